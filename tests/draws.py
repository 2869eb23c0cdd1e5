"""Test helper: the product's random-draw layout, restated with numpy (from
the oracle's Philox) and on the GPU with torch (from moea_rng_blocks), and a
reproduction composed from the reference's own kernels fed with those draws.

The product computes every draw in registers from Philox4x32-10 blocks keyed
by (seed, element, generation, tag); `moea_rng_blocks` returns the raw blocks.
This module turns them into the explicit arrays that the reference's kernels
take (candidate pairs, SBX (u1, u2), signs and copy draws, PM (u1, u2)), so a
generation of the product can be checked bit for bit against
mating_selection.cu:11-35, sbx_crossover.cu:20-70 and
polynomial_mutation.cu:20-60 run on the same numbers.

Layout (tags: 2 mating, 3 crossover, 4 mutation, 5 crossover test, 6 copy):
  mating, child i:       block (i, 2): a = w0 % active, b = w1 % active
  crossover, pair p, variables 4j .. 4j+3: block b = p * ceil(D/4) + j of
                         tag 3, word i for variable 4j+i: u1 = unit(w),
                         sign = w & 1; u2 from block b of tag 5 only when
                         sbx_prob < 1 (else 0), copy from block b of tag 6
                         only when copy_prob > 0 (else 0)
  mutation, child c:     limit = pm_prob / D in FP32; draw k of child c is
                         block k * n + c of tag 4: gap = floor(ln u / ln(1 -
                         limit)) in FP64 with u = ((w0 >> 8) + 1) 2^-24;
                         site = previous site + 1 + gap (start -1), stop at
                         site >= D; the site's amplitude is unit(w1).  In the
                         explicit PM arrays a site has test draw 0 and every
                         other variable test draw 2 (never below the limit).
  unit(w) = (w >> 8) * 2^-24
"""
from __future__ import annotations

import numpy as np
import torch

TAG_MATING, TAG_CROSSOVER, TAG_MUTATION, TAG_CROSS_TEST, TAG_COPY = 2, 3, 4, 5, 6


def _unit_np(w: np.ndarray) -> np.ndarray:
    return (w >> 8).astype(np.float32) * np.float32(1.0 / 16777216.0)


def _u32(blocks: torch.Tensor) -> torch.Tensor:
    """int32 words of moea_rng_blocks as non-negative int64."""
    return blocks.to(torch.int64) & 0xFFFFFFFF


def _unit(w: torch.Tensor) -> torch.Tensor:
    return (w >> 8).to(torch.float32) * (1.0 / 16777216.0)


# ---------------------------------------------------------------- numpy (oracle Philox)
def mating_candidates_np(oracle, seed, generation, n, active):
    w = oracle.philox_stream(seed, generation, TAG_MATING, n)
    return np.stack([w[:, 0] % active, w[:, 1] % active], 1).astype(np.int32)


def _per_variable(blocks: np.ndarray, pairs: int, D: int) -> np.ndarray:
    """(pairs * ceil(D/4), 4) words -> (pairs * D) words, variable order."""
    D4 = (D + 3) // 4
    return blocks.reshape(pairs, D4 * 4)[:, :D].reshape(-1)


def crossover_draws_np(oracle, seed, generation, n, D, sbx_prob, copy_prob):
    """SBX draws of n children: u (pairs*D, 2), sign (pairs*D), copy (pairs*D)."""
    pairs = n // 2
    count = pairs * ((D + 3) // 4)
    w = _per_variable(oracle.philox_stream(seed, generation, TAG_CROSSOVER, count), pairs, D)
    u2 = (_unit_np(_per_variable(oracle.philox_stream(seed, generation, TAG_CROSS_TEST, count), pairs, D))
          if sbx_prob < 1.0 else np.zeros(pairs * D, np.float32))
    copy = (_unit_np(_per_variable(oracle.philox_stream(seed, generation, TAG_COPY, count), pairs, D))
            if copy_prob > 0.0 else np.zeros(pairs * D, np.float32))
    return np.stack([_unit_np(w), u2], 1), (w & 1).astype(np.int32), copy


def _sites(fetch, n, D, pm_prob):
    """Mutation sites of n children: (child, variable, amplitude) lists.
    fetch(k) returns the (n, 4) blocks of draw k of every child."""
    limit = np.float32(pm_prob) / np.float32(D)
    out = []
    if not limit > 0:
        return out
    log_keep = 0.0 if limit >= 1 else float(np.log1p(-np.float64(limit)))
    site = np.full(n, -1, np.int64)
    live = np.ones(n, bool)
    k = 0
    while live.any():
        w = fetch(k)
        if log_keep < 0.0:
            u = ((w[:, 0] >> 8) + 1).astype(np.float64) * (1.0 / 16777216.0)
            gap = np.minimum(np.floor(np.log(u) / log_keep), D).astype(np.int64)
        else:
            gap = np.zeros(n, np.int64)
        site = np.where(live, site + 1 + gap, site)
        live &= site < D
        for c in np.nonzero(live)[0]:
            out.append((int(c), int(site[c]), float(_unit_np(w[c:c + 1, 1])[0])))
        k += 1
    return out


def mutation_draws_np(oracle, seed, generation, n, D, pm_prob):
    """Explicit PM draws (n*D, 2) of the product's mutation sites."""
    def fetch(k):
        return oracle.philox_stream(seed, generation, TAG_MUTATION, (k + 1) * n)[k * n:]
    um = np.zeros((n * D, 2), np.float32)
    um[:, 0] = 2.0
    for c, d, amp in _sites(fetch, n, D, pm_prob):
        um[c * D + d] = (0.0, amp)
    return um


# ---------------------------------------------------------------- torch (product Philox)
def mating_candidates(st, seed: int, generation: int, n: int, active: int) -> torch.Tensor:
    w = _u32(st.rng_blocks(seed, generation, TAG_MATING, n))
    return torch.stack((w[:, 0] % active, w[:, 1] % active), 1).to(torch.int32).contiguous()


def variation_draws(st, seed: int, generation: int, n: int, D: int, sbx_prob: float = 1.0,
                    copy_prob: float = 0.0, pm_prob: float = 1.0):
    """Explicit SBX and PM draws of an offspring population of n children with
    D variables: u (pairs*D, 2), sign (pairs*D), copy (pairs*D) and the PM
    draws (n*D, 2) in child-major order."""
    pairs = n // 2
    D4 = (D + 3) // 4
    dev = "cuda"

    def per_var(tag):
        w = _u32(st.rng_blocks(seed, generation, tag, pairs * D4))
        return w.reshape(pairs, D4 * 4)[:, :D].reshape(-1)
    w = per_var(TAG_CROSSOVER)
    u2 = _unit(per_var(TAG_CROSS_TEST)) if sbx_prob < 1.0 else torch.zeros(pairs * D, device=dev)
    copy = _unit(per_var(TAG_COPY)) if copy_prob > 0.0 else torch.zeros(pairs * D, device=dev)
    u = torch.stack((_unit(w), u2), 1).contiguous()
    sign = (w & 1).to(torch.int32).contiguous()

    def fetch(k):
        return _u32(st.rng_blocks(seed, generation, TAG_MUTATION, (k + 1) * n))[k * n:].cpu().numpy()
    um = torch.zeros((n * D, 2), dtype=torch.float32)
    um[:, 0] = 2.0
    for c, d, amp in _sites(fetch, n, D, pm_prob):
        um[c * D + d, 0] = 0.0
        um[c * D + d, 1] = amp
    return u, sign, copy.contiguous(), um.to(dev).contiguous()


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
    u, sign, copy, um = variation_draws(st, seed, generation, n_off, D, sbx_prob, sbx_copy_prob, pm_prob)
    off = R.sbx_t(parents, pidx, bounds, u, sign, copy, sbx_eta, sbx_prob, sbx_copy_prob, n_off)
    if mutate:
        R.pm_t(off, bounds, um, pm_eta, pm_prob)
    return off, pidx
