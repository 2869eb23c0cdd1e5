"""Test helper: the product's random-draw layout, restated on the GPU with
torch, and a reproduction composed from the reference's own kernels fed with
those draws.

The product computes every draw in registers from Philox4x32-10 blocks keyed
by (seed, element, generation, tag); `moea_rng_blocks` returns the raw blocks.
This module turns them into the explicit arrays that the reference's kernels
take (candidate pairs, SBX (u1, u2), signs and copy draws, PM (u1, u2)), so a
generation of the product can be checked bit for bit against
mating_selection.cu:11-35, sbx_crossover.cu:20-70 and
polynomial_mutation.cu:20-60 run on the same numbers.

Layout (tags: 2 mating, 3 crossover, 4 mutation):
  mating, child i:        block (i, 2): a = w0 % active, b = w1 % active
  variation, element e:   e = p*D + d for pair p (the last child of an odd
                          population is p = pairs); block (e, 3):
                            SBX u1 = unit(w0), sign = w0 & 1, u2 = unit(w1),
                            copy = unit(w2);
                            PM test draw of child 2p = unit(w3), of child
                            2p+1 = unit(low bytes of w1, w2, w3)
                          block (e, 4), only where a child mutates:
                            PM u2 of child 2p = unit(w0), of child 2p+1 = unit(w1)
  unit(w) = (w >> 8) * 2^-24
"""
from __future__ import annotations

import torch

TAG_MATING, TAG_CROSSOVER, TAG_MUTATION = 2, 3, 4


def _u32(blocks: torch.Tensor) -> torch.Tensor:
    """int32 words of moea_rng_blocks as non-negative int64."""
    return blocks.to(torch.int64) & 0xFFFFFFFF


def _unit(w: torch.Tensor) -> torch.Tensor:
    return (w >> 8).to(torch.float32) * (1.0 / 16777216.0)


def mating_candidates(st, seed: int, generation: int, n: int, active: int) -> torch.Tensor:
    w = _u32(st.rng_blocks(seed, generation, TAG_MATING, n))
    return torch.stack((w[:, 0] % active, w[:, 1] % active), 1).to(torch.int32).contiguous()


def variation_draws(st, seed: int, generation: int, n: int, D: int):
    """Explicit SBX and PM draws of an offspring population of n children with
    D variables: u (pairs*D, 2), sign (pairs*D), copy (pairs*D) and the PM
    draws (n*D, 2) in child-major order."""
    pairs = n // 2
    units = pairs + (n & 1)
    w = _u32(st.rng_blocks(seed, generation, TAG_CROSSOVER, units * D))
    m = _u32(st.rng_blocks(seed, generation, TAG_MUTATION, units * D))
    sbx = w[: pairs * D]
    u = torch.stack((_unit(sbx[:, 0]), _unit(sbx[:, 1])), 1).contiguous()
    sign = (sbx[:, 0] & 1).to(torch.int32).contiguous()
    copy = _unit(sbx[:, 2]).contiguous()
    low = ((w[:, 1] & 0xFF) << 24) | ((w[:, 2] & 0xFF) << 16) | ((w[:, 3] & 0xFF) << 8)
    test_a = _unit(w[:, 3]).view(units, D)
    test_b = _unit(low).view(units, D)
    amp_a = _unit(m[:, 0]).view(units, D)
    amp_b = _unit(m[:, 1]).view(units, D)
    um = torch.empty((units * 2, D, 2), dtype=torch.float32, device=w.device)
    um[0::2, :, 0], um[0::2, :, 1] = test_a, amp_a
    um[1::2, :, 0], um[1::2, :, 1] = test_b, amp_b
    return u, sign, copy, um[:n].reshape(n * D, 2).contiguous()


def reference_reproduce(st, R, parents, cv, rank, active, bounds, n_off, *, mating, seed, generation,
                        sbx_eta, sbx_prob, sbx_copy_prob, pm_eta, pm_prob, mutate=True):
    """Offspring from the reference's tournament, SBX and PM kernels on the
    product's draws.  mating 1 = tournament, 0 = random."""
    n_par, D = parents.shape
    cand = mating_candidates(st, seed, generation, n_off, active)
    if mating == 1:
        pidx = torch.from_numpy(R.tournament(cand.cpu().numpy(), rank.cpu().numpy(), cv.cpu().numpy())).cuda()
    else:
        pidx = cand[:, 0].contiguous()
    u, sign, copy, um = variation_draws(st, seed, generation, n_off, D)
    off = R.sbx_t(parents, pidx, bounds, u, sign, copy, sbx_eta, sbx_prob, sbx_copy_prob, n_off)
    if mutate:
        R.pm_t(off, bounds, um, pm_eta, pm_prob)
    return off, pidx
