"""Build libdgop.so (the sm_100a kernels and the C ABI) in-tree with nvcc.

    python -m gendil_b200.build [--fast] [--jobs N] [--clean]

Objects go to ``gendil_b200/_build/<variant>/``; each object is rebuilt only when its source,
the package headers or the flags change.  ``--fast`` (or DGOP_FAST_BUILD=1) compiles only the
(dimension, order, quadrature) shapes the tests and benchmark workloads use.

Every unit is compiled for sm_100a.  The hot-path units (Kronecker kernel, Krylov kernels, C ABI)
and the fast build carry -lineinfo; the full build's generic instantiation units (several hundred
kernels) do not, which keeps the library about three times smaller.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import hashlib
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
INCLUDE = os.path.join(ROOT, "include")
LIB = os.path.join(PKG, "libdgop.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
BASE_FLAGS = ["-std=c++17", "-O3", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
              "-I" + INCLUDE, "-I" + CSRC] + ARCH

# Non-instantiation sources; gen_generic.cu is compiled once per (dimension, N).
SOURCES = ["dgop_api.cu", "registry.cu", "basis.cpp", "kron_plan.cpp", "gen_kron3d.cu", "krylov.cu", "host_io.cu", "batch.cu", "batch_solve.cu", "sipdg.cu"]


def nvcc():
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _headers_digest():
    h = hashlib.sha256()
    for d in (CSRC, INCLUDE):
        for name in sorted(os.listdir(d)):
            if name.endswith((".h", ".cuh", ".hpp")):
                with open(os.path.join(d, name), "rb") as f:
                    h.update(name.encode())
                    h.update(f.read())
    return h.hexdigest()


def _deps_digest(cc, src, flags):
    """Digest of the package headers a unit includes (from nvcc -M), so a header change rebuilds
    only the units that use it."""
    cmd = [cc] + flags + (["-x", "cu"] if src.endswith(".cpp") else []) + ["-M", src]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        return _headers_digest()
    deps = sorted({t for t in r.stdout.replace("\\\n", " ").split() if t.startswith(ROOT) and not t.endswith(":")})
    h = hashlib.sha256()
    for d in deps:
        if os.path.isfile(d):
            with open(d, "rb") as f:
                h.update(d.encode())
                h.update(f.read())
    return h.hexdigest()


def _jobs(fast):
    jobs = []
    for src in SOURCES:
        path = os.path.join(CSRC, src)
        if not os.path.exists(path):
            raise FileNotFoundError(f"listed source {src} is missing from {CSRC}")
        jobs.append((src, path, []))
    gnd = os.path.join(CSRC, "gen_kronnd.cu")
    for d in range(1, 7):
        jobs.append((f"gen_kronnd_d{d}.cu", gnd, [f"-DDGOP_GEN_D={d}"]))
    gen = os.path.join(CSRC, "gen_generic.cu")
    for d in range(1, 7):
        for n in range(1, 9):
            jobs.append((f"gen_generic_d{d}_n{n}.cu", gen, [f"-DDGOP_GEN_D={d}", f"-DDGOP_GEN_N={n}"]))
    return jobs


def build(fast=None, jobs=None, clean=False, verbose=False):
    if fast is None:
        fast = os.environ.get("DGOP_FAST_BUILD", "0") not in ("", "0")
    variant = "fast" if fast else "full"
    out_dir = os.path.join(PKG, "_build", variant)
    if clean and os.path.isdir(out_dir):
        shutil.rmtree(out_dir)
    os.makedirs(out_dir, exist_ok=True)
    flags = BASE_FLAGS + (["-DDGOP_FAST_BUILD"] if fast else [])
    cc = nvcc()
    work = _jobs(fast)

    def compile_one(job):
        name, src, extra = job
        if fast or not name.startswith("gen_generic"):
            extra = ["-lineinfo"] + extra
        obj = os.path.join(out_dir, name.rsplit(".", 1)[0] + ".o")
        stamp = obj + ".sha"
        h = hashlib.sha256()
        with open(src, "rb") as f:
            h.update(f.read())
        h.update(_deps_digest(cc, src, flags + extra).encode())
        h.update(" ".join(flags + extra).encode())
        digest = h.hexdigest()
        if os.path.exists(obj) and os.path.exists(stamp) and open(stamp).read() == digest:
            return obj, False
        cmd = [cc] + flags + extra + ["-c", src, "-o", obj]
        if src.endswith(".cpp"):
            cmd = [cc] + flags + extra + ["-x", "cu", "-c", src, "-o", obj]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed on {name}:\n{' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
        with open(stamp, "w") as f:
            f.write(digest)
        return obj, True

    njobs = jobs or os.cpu_count() or 4
    objs, rebuilt = [], 0
    with cf.ThreadPoolExecutor(max_workers=njobs) as ex:
        # largest units first
        for obj, did in ex.map(compile_one, sorted(work, key=lambda j: -int("gen" in j[0]))):
            objs.append(obj)
            rebuilt += int(did)
    lib_tmp = LIB + ".tmp"
    link = [cc] + ARCH + ["-shared", "-o", lib_tmp] + objs + ["-lcudart_static", "-lrt", "-lpthread", "-ldl"]
    variant_file = os.path.join(PKG, "libdgop.variant")
    current = open(variant_file).read().strip() if os.path.exists(variant_file) else ""
    if rebuilt or not os.path.exists(LIB) or current != variant:
        r = subprocess.run(link, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{' '.join(link)}\n{r.stdout}\n{r.stderr}")
        os.replace(lib_tmp, LIB)
        with open(variant_file, "w") as f:
            f.write(variant)
    if verbose:
        print(f"libdgop.so ({variant}): {rebuilt} of {len(objs)} objects rebuilt")
    return LIB


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--fast", action="store_true")
    ap.add_argument("--jobs", type=int, default=None)
    ap.add_argument("--clean", action="store_true")
    a = ap.parse_args(argv)
    build(fast=a.fast or None, jobs=a.jobs, clean=a.clean, verbose=True)


if __name__ == "__main__":
    sys.exit(main())
