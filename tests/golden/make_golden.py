"""Generate the golden fixtures of this directory from the reference itself.

Runs the reference's own TPB code (compiled unchanged by ``make -C oracle ref`` into
oracle/_ref/ref_dump, single-rank MPI shim) on small inputs and stores what it produced:
excitation tables, the diagonal, one sigma of a seeded vector, the Davidson energy/vector and
the RDMs.  Large arrays are stored whole when small and as sampled entries plus checksums
otherwise, so the fixtures stay a few MB.  Needs the reference checkout (REF, default
/root/reference); the committed .npz files are what the tests read.

    python tests/golden/make_golden.py [case ...]
"""
from __future__ import annotations

import json
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "sbd-pub_b200", "python"))
import synth  # noqa: E402

REF = os.environ.get("REF", "/root/reference")
DUMP = os.path.join(ROOT, "oracle", "_ref", "ref_dump")


def _synthetic_inputs(tmp, L, na_e, nb_e, na_cnt, nb_cnt, seed):
    h1, eri, core = synth.synthetic_hamiltonian(L, seed)
    fd = os.path.join(tmp, "fcidump.txt")
    synth.write_fcidump(fd, L, na_e + nb_e, h1, eri, core, ms2=na_e - nb_e)
    a = synth.sample_strings(L, na_e, na_cnt, seed=seed + 1)
    b = synth.sample_strings(L, nb_e, nb_cnt, seed=seed + 2)
    fa, fb = os.path.join(tmp, "a.txt"), os.path.join(tmp, "b.txt")
    synth.write_strings(fa, a, L)
    synth.write_strings(fb, b, L)
    return fd, fa, fb


CASES = {
    # name: (inputs, davidson (it, nb, tol), rdm, store_full)
    "n2_1em3": dict(fcidump=f"{REF}/data/n2/fcidump.txt", adet=f"{REF}/data/n2/1em3-alpha.txt",
                    davidson=(10, 10, 1e-8), rdm=True, full=False, lanczos=(2, 40, 1e-8),
                    published=-109.04162110, published_src="data/n2/README.md:5"),
    "h2o_1em3": dict(fcidump=f"{REF}/data/h2o/fcidump.txt", adet=f"{REF}/data/h2o/h2o-1em3-alpha.txt",
                     davidson=(10, 10, 1e-8), rdm=False, full=False,
                     published=-76.23594663, published_src="data/h2o/README.md:6"),
    # carryover = (ratio, threshold, cutoff) of the carry-over dumps (ref_dump --carryover);
    # lanczos = (iterations, block, tolerance) of a Lanczos run (ref_dump --lanczos)
    "syn8": dict(synthetic=(8, 3, 3, 56, 56, 11), davidson=(10, 10, 1e-10), rdm=True, full=True,
                 carryover=(0.5, 0.01, 1e-3), lanczos=(3, 20, 1e-10)),
    "syn10_ab": dict(synthetic=(10, 4, 3, 120, 90, 23), davidson=(10, 10, 1e-10), rdm=True, full=True,
                     carryover=(0.3, 1e-3, 1e-4), lanczos=(3, 20, 1e-10)),
    "syn12_co": dict(synthetic=(12, 5, 5, 200, 150, 31), davidson=(10, 10, 1e-10), rdm=False, full=True,
                     carryover=(0.25, 1e-4, 1e-5), lanczos=(3, 30, 1e-10)),
    "fci12": dict(synthetic_named="fci12", davidson=(10, 10, 1e-8), rdm=False, full=False),
    # init = (init, seed): Davidson from the reference's seeded random start (--init 1 --seed) instead
    # of the HF determinant; w0 is that start vector as BasisInitVector built it
    "syn8_init1": dict(synthetic=(8, 3, 3, 56, 56, 11), davidson=(30, 10, 1e-10), rdm=False, full=True,
                       init=(1, 1729)),
    "n2_1em3_init1": dict(fcidump=f"{REF}/data/n2/fcidump.txt", adet=f"{REF}/data/n2/1em3-alpha.txt",
                          davidson=(30, 10, 1e-8), rdm=False, full=False, init=(1, 4242)),
    # the benchmark's larger selected-CI workloads (synthetic_named = a synth.CONFIGS entry): sigma
    # of the closed-form vector (ref_dump --sigma_hash), so a test regenerates its input at any size;
    # the 16M- and 100M-determinant sets also carry the reference's FP64 Davidson energy.  Only
    # samples and checksums of the N-vectors are stored.
    "sci24": dict(synthetic_named="sci24", davidson=(40, 10, 1e-6), rdm=False, full=False, sigma_hash=True,
                  dedupe_tables=True),
    "sci32": dict(synthetic_named="sci32", davidson=None, rdm=False, full=False, sigma_hash=True,
                  dedupe_tables=True),
    "sci28": dict(synthetic_named="sci28", davidson=(40, 10, 1e-6), rdm=False, full=False, sigma_hash=True,
                  dedupe_tables=True),
}


def run_case(name: str, spec: dict, out_dir: str):
    with tempfile.TemporaryDirectory() as tmp:
        bdet = None
        if "synthetic" in spec:
            fd, fa, fb = _synthetic_inputs(tmp, *spec["synthetic"])
            bdet = fb
        elif "synthetic_named" in spec:
            L, n, cnt = synth.CONFIGS[spec["synthetic_named"]]
            h1, eri, core = synth.synthetic_hamiltonian(L)
            fd = os.path.join(tmp, "fcidump.txt")
            fa = os.path.join(tmp, "a.txt")
            synth.write_fcidump(fd, L, 2 * n, h1, eri, core)
            synth.write_strings(fa, synth.sample_strings(L, n, cnt), L)
        else:
            fd, fa = spec["fcidump"], spec["adet"]
        cmd = [DUMP, "--fcidump", fd, "--adetfile", fa, "--out", tmp]
        cmd += ["--sigma_hash"] if spec.get("sigma_hash") else ["--sigma_seed", "7"]
        if bdet:
            cmd += ["--bdetfile", bdet]
        if spec["davidson"]:
            it, nb, tol = spec["davidson"]
            cmd += ["--davidson", str(it), str(nb), repr(tol)]
        if "init" in spec:
            cmd += ["--init", str(spec["init"][0]), str(spec["init"][1])]
        if spec["rdm"]:
            cmd += ["--rdm"]
        if "carryover" in spec:
            cmd += ["--carryover"] + [repr(v) for v in spec["carryover"]]
        if "lanczos" in spec:
            cmd += ["--lanczos"] + [repr(v) for v in spec["lanczos"]]
        env = dict(os.environ, OMP_NUM_THREADS=str(os.cpu_count()))
        out = subprocess.run(cmd, check=True, env=env, capture_output=True, text=True).stdout
        lanczos_lines = sum(1 for l in out.splitlines() if l.startswith(" Lanczos iteration"))
        L = synth.read_fcidump(fd)[0]
        rd = lambda f, dt=np.float64: np.fromfile(os.path.join(tmp, f), dtype=dt)  # noqa: E731
        astr, bstr = rd("astr.u64", np.uint64), rd("bstr.u64", np.uint64)
        n = len(astr) * len(bstr)
        rng = np.random.default_rng(0)
        idx = np.unique(rng.integers(0, n, size=min(n, 512)))
        data = dict(astr=astr, bstr=bstr, idx=idx)
        tasks = [list(map(int, l.split())) for l in open(os.path.join(tmp, "tasks.txt"))]
        data["tasks"] = np.array(tasks, dtype=np.int64)
        # task 0 = type 2 (alpha singles, doubles); task 1 = type 1 (beta); task 2 = type 0
        for t, kinds in ((0, ("sa", "da")), (1, ("sb", "db")), (2, ("sa", "sb"))):
            for k in kinds:
                off = rd(f"task{t}_{k}_off.u64", np.uint64)
                ket = rd(f"task{t}_{k}_ket.u64", np.uint64).astype(np.uint32)
                cran = rd(f"task{t}_{k}_cran.i32", np.int32).astype(np.int8)
                data[f"t{t}_{k}_off"] = off
                data[f"t{t}_{k}_ket"] = ket
                data[f"t{t}_{k}_cran"] = cran
        if spec.get("dedupe_tables") and np.array_equal(astr, bstr):
            # identical string lists: every task's tables are task 0's, except that the CrAn labels
            # of beta entries are the alpha ones + 1 (spin orbital 2p + spin); checked here, one copy kept
            same = {("t1", "sb"): "sa", ("t1", "db"): "da", ("t2", "sa"): "sa", ("t2", "sb"): "sa"}
            for (t, k), k0 in same.items():
                for part in ("off", "ket", "cran"):
                    ref = data[f"t0_{k0}_{part}"]
                    if part == "cran" and k[1] == "b":
                        ref = ref + 1
                    assert np.array_equal(data.pop(f"{t}_{k}_{part}"), ref), (t, k, part)
            data["tables_deduped"] = np.array([1])
        for vec in ("hii", "sigma_in", "sigma_out", "W", "w0"):
            if vec == "W" and not spec["davidson"]:
                continue
            if vec == "w0" and "init" not in spec:
                continue
            v = rd(f"{vec}.f64")
            if spec["full"]:
                data[vec] = v
            data[vec + "_sample"] = v[idx]
            data[vec + "_sum"] = np.array([v.sum(), (v * v).sum(), np.abs(v).sum()])
        if spec["davidson"]:
            data["energy"] = np.array([float(open(os.path.join(tmp, "davidson.txt")).read())])
        if spec["rdm"]:
            r1, r2 = rd("rdm1.f64"), rd("rdm2.f64")
            data["rdm1"] = r1
            if spec["full"]:
                data["rdm2"] = r2
            ridx = np.unique(rng.integers(0, len(r2), size=min(len(r2), 4096)))
            data["rdm2_idx"] = ridx
            data["rdm2_sample"] = r2[ridx]
            data["rdm2_sum"] = np.array([r2.sum(), (r2 * r2).sum(), np.abs(r2).sum()])
        if "carryover" in spec:
            # carry-over strings of W: co1 (threshold), co1r (ratio), co2 (co1 + singles; equal
            # electron counts only), co3 (singles of determinants above the cutoff)
            for tag in ("co1", "co1r", "co2", "co3"):
                for s_ in ("a", "b"):
                    f = os.path.join(tmp, f"{tag}_{s_}.u64")
                    if os.path.exists(f):
                        data[f"{tag}_{s_}"] = np.fromfile(f, dtype=np.uint64)
            vals = [float(x) for x in open(os.path.join(tmp, "carryover.txt")).read().split()]
            data["carryover"] = np.array(vals)  # ratio, threshold, cutoff, truncated a/b, total
        if "lanczos" in spec:
            # energy <W|H|W> after the reference's Lanczos and how many step lines it printed
            data["lanczos"] = np.array([float(open(os.path.join(tmp, "lanczos.txt")).read()), lanczos_lines])
            if spec["full"]:
                data["W_lanczos"] = rd("W_lanczos.f64")
        # the integrals as the reference's SetupIntegrals holds them (h1, packed store, core)
        _, _, h1, eri, core = synth.read_fcidump(fd)
        data["h1"], data["eri"], data["core"] = h1, eri, np.array([core])
        np.savez_compressed(os.path.join(out_dir, f"{name}.npz"), **data)
        meta = dict(norb=L, na=len(astr), nb=len(bstr), rdm=spec["rdm"], full=spec["full"],
                    davidson=list(spec["davidson"]) if spec["davidson"] else None)
        if spec["davidson"]:
            meta["energy"] = float(data["energy"][0])
        if spec.get("sigma_hash"):
            meta["sigma_input"] = "hash"
        for k in ("published", "published_src"):
            if k in spec:
                meta[k] = spec[k]
        if "fcidump" in spec:
            meta["fcidump"] = os.path.relpath(spec["fcidump"], REF)
            meta["adet"] = os.path.relpath(spec["adet"], REF)
        if "synthetic" in spec:
            meta["synthetic"] = list(spec["synthetic"])
        if "synthetic_named" in spec:
            meta["synthetic_named"] = spec["synthetic_named"]
        if "carryover" in spec:
            meta["carryover"] = list(spec["carryover"])
        if "lanczos" in spec:
            meta["lanczos"] = list(spec["lanczos"])
        if "init" in spec:
            meta["init"] = list(spec["init"])
        return meta


def write_bin_strings(path, strings, L, rng):
    """Binary string file as DecodeAlphaDets reads it: ceil(L/8)-byte big-endian records, the
    string in the low L bits, random bits in the unused high bits (which the reader skips)."""
    rb = (L + 7) // 8
    with open(path, "wb") as f:
        for s in strings:
            pad = int(rng.integers(0, 1 << (8 * rb - L))) << L if 8 * rb > L else 0
            f.write((int(s) | pad).to_bytes(rb, "big"))


def make_strings_fixture(out_dir):
    """tests/golden/strings.npz: text and binary string files (unsorted, with duplicates, CRLF
    line ends in one of them) and the strings the reference's LoadAlphaDets makes of them
    (astr.u64 of ref_dump: from_string / DecodeAlphaDets, then sort_bitarray)."""
    rng = np.random.default_rng(4242)
    data, meta = {}, {}
    for L, ne, cnt in ((12, 5, 300), (20, 7, 400), (36, 9, 500)):
        pool = synth.sample_strings(L, ne, cnt, seed=L)
        strs = [int(pool[i]) for i in rng.integers(0, len(pool), size=cnt + cnt // 3)]  # duplicates
        with tempfile.TemporaryDirectory() as tmp:
            h1, eri, core = synth.synthetic_hamiltonian(L, seed=L)
            fd = os.path.join(tmp, "fcidump.txt")
            synth.write_fcidump(fd, L, 2 * ne, h1, eri, core)
            ftxt, fbin = os.path.join(tmp, "a.txt"), os.path.join(tmp, "a.bin")
            eol = "\r\n" if L == 20 else "\n"
            with open(ftxt, "w", newline="") as f:
                for s_ in strs:
                    f.write(format(s_, f"0{L}b") + eol)
            write_bin_strings(fbin, strs, L, rng)
            for kind, path in (("txt", ftxt), ("bin", fbin)):
                d = os.path.join(tmp, kind)
                os.makedirs(d)
                subprocess.run([DUMP, "--fcidump", fd, "--adetfile", path, "--out", d], check=True,
                               stdout=subprocess.DEVNULL)
                data[f"L{L}_{kind}_bytes"] = np.frombuffer(open(path, "rb").read(), np.uint8)
                data[f"L{L}_{kind}_ref"] = np.fromfile(os.path.join(d, "astr.u64"), np.uint64)
        meta[f"L{L}"] = dict(electrons=ne, lines=len(strs), unique=int(len(set(strs))))
    np.savez_compressed(os.path.join(out_dir, "strings.npz"), **data)
    return meta


# Larger selected sets of the reference's data directories with the energies its READMEs publish
# (8 decimals).  The Hamiltonians are those of the h2o_1em3 / n2_1em3 fixtures (same FCIDUMP).
PUBLISHED = {
    "h2o_1em4": ("h2o_1em3", "data/h2o/h2o-1em4-alpha.txt", -76.24295848, "data/h2o/README.md:7"),
    "h2o_1em5": ("h2o_1em3", "data/h2o/h2o-1em5-alpha.txt", -76.24373504, "data/h2o/README.md:8"),
    "h2o_1em6": ("h2o_1em3", "data/h2o/h2o-1em6-alpha.txt", -76.24377593, "data/h2o/README.md:9"),
    "h2o_1em7": ("h2o_1em3", "data/h2o/h2o-1em7-alpha.txt", -76.24377678, "data/h2o/README.md:10"),
    "n2_3em4": ("n2_1em3", "data/n2/3em4-alpha.txt", -109.04697304, "data/n2/README.md:7"),
    "n2_1em4": ("n2_1em3", "data/n2/1em4-alpha.txt", -109.04835269, "data/n2/README.md:8"),
    "n2_1em5": ("n2_1em3", "data/n2/1em5-alpha.txt", -109.04871934, "data/n2/README.md:10"),
    "n2_1em6": ("n2_1em3", "data/n2/1em6-alpha.txt", -109.04874139, "data/n2/README.md:12"),
}


def make_published_fixture(out_dir):
    """tests/golden/published.npz: the string sets of PUBLISHED, read by the oracle's LoadAlphaDets
    restatement (orc_load_strings, held equal to the reference's reader by tests/test_strings.py),
    and their published energies in the index."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle
    data, meta = {}, {}
    for name, (base, adet, energy, src) in PUBLISHED.items():
        L = json.load(open(os.path.join(HERE, "cases.json")))[base]["norb"]
        a = pyoracle.load_strings(os.path.join(REF, adet), L)
        data[f"{name}_astr"] = a
        meta[name] = dict(base=base, adet=adet, published=energy, published_src=src, na=int(len(a)),
                          ndet=int(len(a)) ** 2)
    np.savez_compressed(os.path.join(out_dir, "published.npz"), **data)
    return meta


def main():
    names = sys.argv[1:] or list(CASES) + ["strings", "published"]
    index_path = os.path.join(HERE, "cases.json")
    index = json.load(open(index_path)) if os.path.exists(index_path) else {}
    if "strings" in names:
        names = [n for n in names if n != "strings"]
        print("case strings", flush=True)
        index["strings"] = make_strings_fixture(HERE)
        json.dump(index, open(index_path, "w"), indent=1, sort_keys=True)
    if "published" in names:
        names = [n for n in names if n != "published"]
        print("case published", flush=True)
        index["published"] = make_published_fixture(HERE)
        json.dump(index, open(index_path, "w"), indent=1, sort_keys=True)
    for name in names:
        print("case", name, flush=True)
        index[name] = run_case(name, CASES[name], HERE)
        json.dump(index, open(index_path, "w"), indent=1, sort_keys=True)


if __name__ == "__main__":
    main()
