"""Builds problem plugins against the plugin SDK and caches the results.

A plugin source directory holds .cu / .cpp files (headers beside them) that
implement IProblemEvaluator and register it with CUDA_MOEA_REGISTER_PROBLEM.
``build_problem`` compiles every source file with nvcc against the SDK
headers into one shared library and keeps it in a content-addressed cache:
the key hashes the files' relative names and contents, the SDK headers, the
compiler's version and the flags, so an unchanged plugin is never rebuilt and
a cache built on one machine is reused on another with the same toolchain.
Finished builds are published by one rename, under a lock, and never change
afterwards.  Runtime parameter values do not enter the key.

Same entry points as the reference's cuda_moea._native_build
(build_problem, clear_cache, export_problem, sdk_directory, cache_directory);
the reference drives CMake, this builder calls nvcc directly.
"""
from __future__ import annotations

import concurrent.futures as cf
import fcntl
import hashlib
import json
import os
import shutil
import subprocess
import tempfile
from contextlib import contextmanager
from pathlib import Path

_SOURCE_SUFFIXES = {".cu", ".cpp", ".cc", ".cxx"}
_SKIP_DIRS = {".git", "__pycache__", "build"}


def sdk_directory() -> Path:
    """Root of the plugin SDK (its headers are under include/)."""
    return Path(__file__).resolve().parent.parent / "sdk"


def cache_directory() -> Path:
    """MOEA_B200_NATIVE_CACHE, else $XDG_CACHE_HOME/moea_b200/native."""
    default = Path(os.environ.get("XDG_CACHE_HOME", Path.home() / ".cache")) / "moea_b200" / "native"
    return Path(os.environ.get("MOEA_B200_NATIVE_CACHE", default)).expanduser().resolve()


def _nvcc() -> str:
    return os.environ.get("NVCC", shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc")


def _tree(root: Path) -> list[Path]:
    files = []
    for dirpath, dirs, names in os.walk(root):
        dirs[:] = sorted(d for d in dirs if d not in _SKIP_DIRS and not d.startswith("."))
        for name in sorted(names):
            files.append(Path(dirpath) / name)
    return files


def _digest(files: list[Path], root: Path, h) -> None:
    for f in files:
        h.update(str(f.relative_to(root)).encode() + b"\0")
        h.update(f.read_bytes())
        h.update(b"\0")


@contextmanager
def _lock(cache: Path):
    cache.mkdir(parents=True, exist_ok=True)
    with (cache / ".lock").open("a") as stream:
        fcntl.flock(stream, fcntl.LOCK_EX)
        try:
            yield
        finally:
            fcntl.flock(stream, fcntl.LOCK_UN)


def _compiler_version(nvcc: str) -> str:
    try:
        return subprocess.run([nvcc, "--version"], capture_output=True, text=True, check=True).stdout
    except (OSError, subprocess.CalledProcessError):
        return ""


def build_problem(source_dir, *, mode: str = "auto", cache_dir=None, architectures: str | None = None,
                  debug: bool = False, force: bool = False, verbose: bool = False,
                  dependencies=(), jobs: int | None = None) -> Path:
    """Path of the plugin library for ``source_dir``, compiling on a cache miss.

    mode "never" only looks the library up (FileNotFoundError when absent);
    ``dependencies`` are extra include directories (hashed with the sources);
    ``architectures`` defaults to MOEA_B200_NATIVE_ARCH or "100a"."""
    if mode not in ("auto", "never"):
        raise ValueError("mode must be 'auto' or 'never'")
    source = Path(source_dir).expanduser().resolve()
    if not source.is_dir():
        raise FileNotFoundError(f"source_dir {source} is not a directory")
    cache = Path(cache_dir).expanduser().resolve() if cache_dir else cache_directory()
    if cache == source or source in cache.parents:
        raise ValueError("cache_dir must be outside source_dir")
    files = _tree(source)
    sources = [f for f in files if f.suffix in _SOURCE_SUFFIXES]
    if not sources:
        raise ValueError(f"no .cu/.cpp sources in {source}")
    arch = architectures or os.environ.get("MOEA_B200_NATIVE_ARCH", "100a")
    deps = [Path(d).expanduser().resolve() for d in dependencies]
    nvcc = _nvcc()
    flags = ["-std=c++17", "-Xcompiler", "-fPIC", "-gencode", f"arch=compute_{arch},code=sm_{arch}",
             "-lineinfo"] + (["-O0", "-g"] if debug else ["-O3"])
    h = hashlib.sha256()
    h.update(json.dumps({"flags": flags, "compiler": _compiler_version(nvcc)}, sort_keys=True).encode())
    _digest(files, source, h)
    sdk_include = sdk_directory() / "include"
    _digest(_tree(sdk_include), sdk_include, h)
    for d in deps:
        _digest(_tree(d), d, h)
    key = h.hexdigest()[:32]
    with _lock(cache):
        final = cache / "artifacts" / key
        library = final / "problem.so"
        if library.is_file() and not force:
            return library
        if mode == "never":
            raise FileNotFoundError("no cached build of this native problem; build it with "
                                    "'python -m cuda_moea.native build SOURCE' or use build='auto'")
        (cache / "work").mkdir(exist_ok=True)
        work = Path(tempfile.mkdtemp(prefix=f"{key}-", dir=cache / "work"))
        try:
            includes = ["-I", str(sdk_include), "-I", str(source)]
            for d in deps:
                includes += ["-I", str(d)]
            log = []

            def compile_one(i_src):
                i, src = i_src
                obj = work / f"{i:04d}_{src.stem}.o"
                cmd = [nvcc, *flags, *includes, "-c", str(src), "-o", str(obj)]
                res = subprocess.run(cmd, capture_output=True, text=True)
                return obj, cmd, res

            with cf.ThreadPoolExecutor(max_workers=jobs or os.cpu_count() or 4) as ex:
                results = list(ex.map(compile_one, enumerate(sources)))
            for obj, cmd, res in results:
                log.append(" ".join(cmd) + "\n" + res.stdout + res.stderr)
                if verbose:
                    print(log[-1])
                if res.returncode != 0:
                    raise RuntimeError(f"native problem build failed:\n{log[-1]}")
            out = work / "problem.so"
            link = [nvcc, "-shared", "-gencode", f"arch=compute_{arch},code=sm_{arch}", "-o", str(out),
                    *[str(r[0]) for r in results]]
            res = subprocess.run(link, capture_output=True, text=True)
            log.append(" ".join(link) + "\n" + res.stdout + res.stderr)
            if res.returncode != 0:
                raise RuntimeError(f"native problem link failed:\n{log[-1]}")
            staging = work / "publish"
            staging.mkdir()
            shutil.copy2(out, staging / "problem.so")
            (staging / "build.log").write_text("\n".join(log))
            (staging / "artifact.json").write_text(json.dumps(
                {"key": key, "source": str(source), "architectures": arch, "debug": debug,
                 "sources": [str(s.relative_to(source)) for s in sources]}, indent=2, sort_keys=True))
            final.parent.mkdir(parents=True, exist_ok=True)
            if final.exists():  # force: replace the old build
                shutil.rmtree(final)
            staging.rename(final)
        finally:
            shutil.rmtree(work, ignore_errors=True)
        return library


def clear_cache(cache_dir=None) -> None:
    """Removes every cached build (stop the processes that use them first)."""
    cache = Path(cache_dir).expanduser().resolve() if cache_dir else cache_directory()
    with _lock(cache):
        for name in ("artifacts", "work"):
            path = cache / name
            if path.exists():
                shutil.rmtree(path)


def export_problem(library, destination) -> Path:
    """Copies a cached build (problem.so and artifact.json) into a new directory."""
    library = Path(library).expanduser().resolve()
    destination = Path(destination).expanduser().resolve()
    destination.mkdir(parents=True, exist_ok=True)
    for name in ("problem.so", "artifact.json"):
        if (destination / name).exists():
            raise FileExistsError(f"{destination / name} exists; choose a new directory")
    shutil.copy2(library, destination / "problem.so")
    if (library.parent / "artifact.json").exists():
        shutil.copy2(library.parent / "artifact.json", destination / "artifact.json")
    return destination / "problem.so"

