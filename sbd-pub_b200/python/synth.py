"""Synthetic TPB problems and FCIDUMP / string-file I/O.

The benchmark problems are seeded synthetic stand-ins with the shapes of the reference's
molecular inputs (the reference's own data/ FCIDUMPs are used as known-answer fixtures by the
tests instead):

* one-electron  h_pp = -2 + 4p/L,  h_pq ~ N(0, 0.05^2) symmetric (p != q);
* two-electron  (pq|rs) = sum_{Lam < 2L} B^Lam_pq B^Lam_rs with B^Lam symmetric, entries
  N(0, 0.1^2) plus 0.5 on the diagonal (so (pp|qq) > 0), 8-fold symmetric, core energy 0;
* strings       the Hartree-Fock string (lowest n orbitals) plus strings drawn without
  replacement with weight 0.3^k, k = excitation rank from HF, sorted ascending; all C(L, n)
  strings when the count reaches it.

Seeds: integrals 1729, strings 137.  FCIDUMP text follows the layout framework/fcidump.h:29-141
reads (header with NORB/NELEC/MS2, "&END", then "value i j k l" lines, 1-based, 0 0 0 0 = core).
"""
from __future__ import annotations

import math
import os

import numpy as np

INTEGRAL_SEED = 1729
STRING_SEED = 137

# Workloads: name -> (norb, electrons per spin, strings per spin)
CONFIGS = {
    "fci12": (12, 6, 924),        # full CI, 853,776 determinants
    "sci24": (24, 8, 4000),       # 16M determinants
    "sci32": (32, 10, 20000),     # 400M determinants
    "sci28": (28, 9, 10000),      # 100M determinants
    "sci36": (36, 12, 40000),     # 1.6B determinants
}


def pair_index(i: int, j: int) -> int:
    a, b = max(i, j), min(i, j)
    return a * (a + 1) // 2 + b


def packed_size(L: int) -> int:
    B = L * (L + 1) // 2
    return B * (B + 1) // 2


def pack_eri(eri: np.ndarray) -> np.ndarray:
    """Dense (pq|rs) [L,L,L,L] -> the 8-fold packed store (basic/integrals.h:64-107)."""
    L = eri.shape[0]
    iu = np.array([(i, j) for i in range(L) for j in range(i + 1)])  # pair index order
    M = eri[iu[:, 0], iu[:, 1]][:, iu[:, 0], iu[:, 1]]  # [B, B]
    B = M.shape[0]
    a, b = np.tril_indices(B)
    out = np.zeros(packed_size(L))
    out[a * (a + 1) // 2 + b] = M[a, b]
    return out


def unpack_eri(store: np.ndarray, L: int) -> np.ndarray:
    idx = np.array([[pair_index(i, j) for j in range(L)] for i in range(L)])
    P = idx.reshape(-1)
    a = np.maximum(P[:, None], P[None, :])
    b = np.minimum(P[:, None], P[None, :])
    return store[a * (a + 1) // 2 + b].reshape(L, L, L, L)


def synthetic_hamiltonian(L: int, seed: int = INTEGRAL_SEED):
    """(h1 [L,L], packed ERI, core) from the seeded generator described in the module doc."""
    rng = np.random.default_rng(seed)
    h1 = np.zeros((L, L))
    iu = np.triu_indices(L, 1)
    off = rng.normal(0.0, 0.05, size=len(iu[0]))
    h1[iu] = off
    h1 = h1 + h1.T
    h1[np.arange(L), np.arange(L)] = -2.0 + 4.0 * np.arange(L) / L
    nlam = 2 * L
    Bm = rng.normal(0.0, 0.1, size=(nlam, L, L))
    Bm = np.triu(Bm) + np.transpose(np.triu(Bm, 1), (0, 2, 1))
    Bm[:, np.arange(L), np.arange(L)] += 0.5
    Bf = Bm.reshape(nlam, L * L)
    eri = (Bf.T @ Bf).reshape(L, L, L, L)
    return h1, pack_eri(eri), 0.0


def sample_strings(L: int, n: int, count: int, seed: int = STRING_SEED) -> np.ndarray:
    """HF plus weighted sampling without replacement (weight 0.3^rank); sorted uint64."""
    total = math.comb(L, n)
    if count >= total:
        from itertools import combinations
        out = [sum(1 << p for p in c) for c in combinations(range(L), n)]
        return np.array(sorted(out), dtype=np.uint64)
    rng = np.random.default_rng(seed)
    kmax = min(n, L - n)
    ks = np.arange(0, kmax + 1)
    w = np.array([math.comb(n, k) * math.comb(L - n, k) * 0.3 ** k for k in ks])
    w /= w.sum()
    hf = (1 << n) - 1
    chosen = {hf}
    while len(chosen) < count:
        batch = min(4 * (count - len(chosen)) + 64, 1 << 16)
        kk = rng.choice(ks, size=batch, p=w)
        for k in kk:
            if k == 0:
                continue
            holes = rng.choice(n, size=k, replace=False)
            parts = rng.choice(L - n, size=k, replace=False) + n
            s = hf
            for h in holes:
                s &= ~(1 << int(h))
            for p in parts:
                s |= 1 << int(p)
            chosen.add(s)
            if len(chosen) >= count:
                break
    return np.array(sorted(chosen), dtype=np.uint64)


def make_problem(name: str, nstrings: int | None = None):
    """Problem for a named workload (optionally with fewer strings, for parity-size cases)."""
    from sbd_tpb import Problem
    L, n, cnt = CONFIGS[name]
    if nstrings is not None:
        cnt = nstrings
    h1, eri, core = synthetic_hamiltonian(L)
    s = sample_strings(L, n, cnt)
    return Problem(norb=L, nelec=2 * n, core=core, h1=h1, eri_packed=eri, astr=s, bstr=s.copy())


def write_fcidump(path: str, L: int, nelec: int, h1: np.ndarray, eri_packed: np.ndarray,
                  core: float = 0.0, ms2: int = 0):
    with open(path, "w") as f:
        f.write(f" &FCI NORB={L},NELEC={nelec},MS2={ms2},\n")
        f.write("  ORBSYM=" + ",".join(["1"] * L) + ",\n  ISYM=1,\n &END\n")
        for i in range(L):
            for j in range(i + 1):
                ij = pair_index(i, j)
                for k in range(L):
                    for l in range(k + 1):
                        kl = pair_index(k, l)
                        if kl > ij:
                            continue
                        v = eri_packed[ij * (ij + 1) // 2 + kl]
                        if v != 0.0:
                            f.write(f" {v:.17g} {i + 1} {j + 1} {k + 1} {l + 1}\n")
        for i in range(L):
            for j in range(i + 1):
                if h1[i, j] != 0.0:
                    f.write(f" {h1[i, j]:.17g} {i + 1} {j + 1} 0 0\n")
        f.write(f" {core:.17g} 0 0 0 0\n")


def read_fcidump(path: str):
    """(L, nelec, h1, packed ERI, core) as framework/fcidump.h + SetupIntegrals read them."""
    header = ""
    ints = []
    in_header = True
    with open(path) as f:
        for line in f:
            line = line.rstrip("\r\n")
            if not line or line[0] == "!":
                continue
            if in_header:
                if "&END" in line:
                    in_header = False
                    continue
                header += line.replace("&FCI", "", 1)
            else:
                t = line.split()
                if len(t) >= 5:
                    ints.append((float(t[0]), int(t[1]), int(t[2]), int(t[3]), int(t[4])))
    kv = {}
    for tok in header.split(","):
        if "=" in tok:
            k, v = tok.split("=", 1)
            kv[k.strip()] = v.strip()
    L = int(kv["NORB"])
    nelec = int(kv.get("NELEC", "0"))
    h1 = np.zeros((L, L))
    eri = np.zeros(packed_size(L))
    core = 0.0
    for v, i, j, k, l in ints:
        if i == j == k == l == 0:
            core = v
        elif k == 0 and l == 0:
            h1[i - 1, j - 1] = v
            h1[j - 1, i - 1] = v
        else:
            a, b = pair_index(i - 1, j - 1), pair_index(k - 1, l - 1)
            a, b = max(a, b), min(a, b)
            eri[a * (a + 1) // 2 + b] = v
    return L, nelec, h1, eri, core


def write_strings(path: str, strs: np.ndarray, L: int):
    with open(path, "w") as f:
        for s in strs:
            s = int(s)
            f.write("".join("1" if (s >> (L - 1 - i)) & 1 else "0" for i in range(L)) + "\n")


def read_strings(path: str, L: int) -> np.ndarray:
    out = set()
    with open(path) as f:
        for line in f:
            line = line.rstrip("\r\n ")
            if not line:
                continue
            v = 0
            for i in range(L):
                if line[L - 1 - i] == "1":
                    v |= 1 << i
            out.add(v)
    return np.array(sorted(out), dtype=np.uint64)


def problem_from_files(fcidump: str, adetfile: str, bdetfile: str | None = None):
    from sbd_tpb import Problem
    L, nelec, h1, eri, core = read_fcidump(fcidump)
    a = read_strings(adetfile, L)
    b = read_strings(bdetfile, L) if bdetfile else a.copy()
    return Problem(norb=L, nelec=nelec, core=core, h1=h1, eri_packed=eri, astr=a, bstr=b)


if __name__ == "__main__":  # write FCIDUMP + string file for a named workload
    import sys
    name, outdir = sys.argv[1], sys.argv[2]
    L, n, cnt = CONFIGS[name]
    h1, eri, core = synthetic_hamiltonian(L)
    os.makedirs(outdir, exist_ok=True)
    write_fcidump(os.path.join(outdir, "fcidump.txt"), L, 2 * n, h1, eri, core)
    write_strings(os.path.join(outdir, "alpha.txt"), sample_strings(L, n, cnt), L)
