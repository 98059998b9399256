"""Generate the golden fixtures of the parity tests from the reference itself.

Runs the reference's own CPU build (oracle/_ref/gtalign, compiled from the
reference sources by oracle/Makefile.ref) on seeded synthetic structure sets
and records, per query-reference pair, what it prints in its JSON output:
TM-scores (5 decimals), RMSD (2 decimals), counts, alignment rows,
secondary-structure rows and the transform.  The input coordinates are
stored with the fixtures, so the tests never need the reference or the
generator again.

For every set the reference is also run a second time with the query moved
by a rigid rotation + translation (which leaves every score unchanged in
exact arithmetic); the agreement between those two reference runs is the
reference's own numerical reproducibility and is stored as `self_agreement`.

    python tests/golden/make_golden.py [set ...]   (needs oracle/_ref/gtalign)

The same sets run by the reference's GPU build (oracle/_ref/gpu/gtalign,
compiled by oracle/Makefile.refgpu; on a machine with a GPU):

    python tests/golden/make_golden.py --gpu --outdir DIR [set ...]

writes DIR/<set>_refgpu.json (its results and self-agreement; the inputs are
those of <set>.npz) and, for every pair both builds report, the agreement
between the reference's GPU and CPU builds.
"""
from __future__ import annotations

import copy
import json
import os
import shutil
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
from gtalign_alpha_b200 import synth  # noqa: E402

BIN = os.path.join(ROOT, "oracle", "_ref", "gtalign")
BIN_GPU = os.path.join(ROOT, "oracle", "_ref", "gpu", "gtalign")

def na_set(seed):
    """Nucleic acids: a query of 3 hairpins, moved noisy copies of it,
    unrelated hairpin chains, and a few proteins (skipped against it).  The
    stems rise 7.5 A per pair, so that a stem residue's only C3' within the
    12.5-15 A pairing window is its partner's (the diagonal neighbours sit
    at 15.7 A): the reference's CPU build picks a partner among several
    candidates with a vectorised reduction whose winner is not always the
    closest one, unlike its GPU form."""
    rng = np.random.default_rng(seed)
    q = synth.na_hairpins(rng, 3, 10, 6, "qry000000", rise=7.5)
    refs = [synth.na_moved_copy(rng, q, float(rng.uniform(0.3, 1.5)), "hom%06d" % k) for k in range(10)]
    refs += [synth.na_hairpins(rng, int(rng.integers(1, 5)), int(rng.integers(5, 13)),
                               int(rng.integers(4, 9)), "ref%06d" % k, rise=7.5) for k in range(14)]
    refs += synth.random_chains(rng, list(rng.integers(60, 200, size=4)), "prt")
    return synth.Workload([q], refs, seed, "nucleic acids")


SETS = {
    # name: (workload builder, reference CLI options)
    "c0_speed13": (lambda: synth.config0(seed=101, n_refs=80, qlen=150),
                   ["--speed=13", "--pre-score=0", "-s", "0"]),
    "c0_default": (lambda: synth.config0(seed=102, n_refs=60, qlen=120),
                   ["--no-detailed-search", "--pre-score=0", "-s", "0"]),
    "c0_filters": (lambda: synth.config0(seed=103, n_refs=60, qlen=180),
                   ["--no-detailed-search"]),  # default --pre-score 0.4 and -s 0.5
    "c0_sym_ref_nodel": (lambda: synth.config0(seed=104, n_refs=40, qlen=100),
                         ["--speed=13", "--pre-score=0", "-s", "0", "--symmetric",
                          "--referenced", "--no-deletions"]),
    # the final stage's phase-2 forms, one set per --refinement code, on
    # homologs of the query only (one clear optimum per pair, so the level's
    # small TM differences show); run with one compute thread: the
    # reference's CPU build stalls intermittently in its full-search levels
    # with several threads
    "c0_level_m1": (lambda: synth.config0(seed=201, n_refs=40, qlen=180, homolog_frac=1.0),
                    ["--no-detailed-search", "--refinement=-1", "--pre-score=0", "-s", "0"], 1),
    "c0_level_0": (lambda: synth.config0(seed=201, n_refs=40, qlen=180, homolog_frac=1.0),
                   ["--no-detailed-search", "--refinement=0", "--pre-score=0", "-s", "0"], 1),
    "c0_level_1": (lambda: synth.config0(seed=201, n_refs=40, qlen=180, homolog_frac=1.0),
                   ["--no-detailed-search", "--refinement=1", "--pre-score=0", "-s", "0"], 1),
    "c0_level_2": (lambda: synth.config0(seed=201, n_refs=40, qlen=180, homolog_frac=1.0),
                   ["--no-detailed-search", "--refinement=2", "--pre-score=0", "-s", "0"], 1),
    "c0_level_3": (lambda: synth.config0(seed=201, n_refs=40, qlen=180, homolog_frac=1.0),
                   ["--no-detailed-search", "--refinement=3", "--pre-score=0", "-s", "0"], 1),
    "c0_2tm": (lambda: synth.config0(seed=109, n_refs=50, qlen=150, homolog_frac=0.5),
               ["--no-detailed-search", "--2tm-score", "--pre-score=0", "-s", "0"]),
    "c0_ssrr": (lambda: synth.config0(seed=110, n_refs=60, qlen=150, homolog_frac=0.5),
                ["--no-detailed-search", "--add-search-by-ss", "--pre-score=0", "-s", "0"]),
    "c0_presim": (lambda: synth.config0(seed=111, n_refs=80, qlen=150, homolog_frac=0.3),
                  ["--no-detailed-search", "--pre-similarity=15", "--pre-score=0", "-s", "0"]),
    "c0_na": (lambda: na_set(112), ["--no-detailed-search", "--pre-score=0", "-s", "0"]),
    # options together: symmetric, referenced, secondary TM-scores, full search
    "c0_combo": (lambda: synth.config0(seed=113, n_refs=50, qlen=140, homolog_frac=0.5),
                 ["--no-detailed-search", "--symmetric", "--referenced", "--2tm-score",
                  "--refinement=2", "--pre-score=0", "-s", "0"], 1),
    "c0_shallow": (lambda: synth.config0(seed=108, n_refs=60, qlen=160),
                   ["--no-detailed-search", "--depth=3", "--pre-score=0.3", "-s", "0.3",
                    "--convergence=6"]),
    # the small configuration at its full size: one 150-residue query against
    # 1,000 targets (lengths U(50,500), 20% homologs), default options (the
    # default --pre-score 0.4 and -s 0.5) without the detailed search, and
    # the --speed=13 preset
    "c0_full": (lambda: synth.config0(seed=1, n_refs=1000, qlen=150), ["--no-detailed-search"]),
    "c0_full_s13": (lambda: synth.config0(seed=1, n_refs=1000, qlen=150), ["--speed=13"]),
    # the spatial-index detailed search: every pair run alone (one query, one
    # reference per call) on one thread, where the reference's fragment slots
    # and score-matrix layout are the pair's own
    "f3_default": (lambda: synth.config0(seed=301, n_refs=60, qlen=150, homolog_frac=0.3),
                   ["--pre-score=0", "-s", "0"], 1, "perpair"),
    "f3_speed12": (lambda: synth.config0(seed=302, n_refs=40, qlen=180, homolog_frac=0.3),
                   ["--speed=12", "--pre-score=0", "-s", "0"], 1, "perpair"),
    "f3_opts": (lambda: synth.config0(seed=303, n_refs=40, qlen=130, homolog_frac=0.3),
                ["--speed=7", "--seedrule=0", "--nbranches=3", "--gapcost=2", "--window=512",
                 "--pre-score=0", "-s", "0"], 1, "perpair"),
    # --depth 1 and 0 (the secondary configuration sections and the extra DP
    # of each branch): --speed 6 and 3 (trigger 50), --speed 0 (trigger 0,
    # 16 branches, --add-search-by-ss)
    "f3_speed6": (lambda: synth.config0(seed=304, n_refs=40, qlen=170, homolog_frac=0.3),
                  ["--speed=6", "--pre-score=0", "-s", "0"], 1, "perpair"),
    "f3_speed3": (lambda: synth.config0(seed=305, n_refs=40, qlen=160, homolog_frac=0.3),
                  ["--speed=3", "--pre-score=0", "-s", "0"], 1, "perpair"),
    "f3_speed0": (lambda: synth.config0(seed=306, n_refs=24, qlen=155, homolog_frac=0.3),
                  ["--speed=0", "--pre-score=0", "-s", "0"], 1, "perpair"),
}


def run_perpair(wl, opts, threads=1, binary=BIN):
    """Each reference in a call of its own (every query against it)."""
    res = {}
    for r in wl.refs:
        res.update(run(synth.Workload(wl.queries, [r], wl.seed), opts, threads, binary))
    return res


def run(wl, opts, threads=8, binary=BIN):
    d = tempfile.mkdtemp(prefix="gtgold")
    try:
        synth.write_dirs(wl, d + "/q", d + "/r")
        subprocess.run([binary, "--qrs=" + d + "/q", "--rfs=" + d + "/r", "-o", d + "/out",
                        "--outfmt=1", "--cpu-threads=%d" % threads, "--cpu-threads-reading=1"] + opts,
                       check=True, capture_output=True)
        res = {}
        for f in os.listdir(d + "/out"):
            J = json.load(open(os.path.join(d, "out", f)))["gtalign_search"]
            qn = os.path.basename(J["query"]["description"].split()[0])[:-4]
            for h in J["search_results"]:
                h = h["hit_record"]
                rn = os.path.basename(h["reference_description"].split()[0])[:-4]
                a = h["alignment"]
                res[qn + "|" + rn] = {
                    "tmq": a["tmscore_query"], "tmr": a["tmscore_refn"], "rmsd": a["rmsd"],
                    "d0q": a["d0_query"], "d0r": a["d0_refn"],
                    "n_identities": a["n_identities"], "n_matched": a["n_matched"],
                    "n_gaps": a["n_gaps"], "n_aligned": a["n_aligned"],
                    "query_from": a["query_from"], "query_to": a["query_to"],
                    "refn_from": a["refn_from"], "refn_to": a["refn_to"],
                    "query_aln": a["query_aln"], "refrn_aln": a["refrn_aln"], "middle": a["middle"],
                    "query_secstr": a["query_secstr"], "refrn_secstr": a["refrn_secstr"],
                    "rotation": h["rotation_matrix_rowmajor"], "translation": h["translation_vector"],
                }
                if "--2tm-score" in opts:
                    res[qn + "|" + rn]["tm2q"] = float(a["2tmscore_query"])
                    res[qn + "|" + rn]["tm2r"] = float(a["2tmscore_refn"])
        return res
    finally:
        shutil.rmtree(d, ignore_errors=True)


def agreement(a, b):
    d, same = [], []
    for k, v in a.items():
        w = b.get(k)
        if w is None:
            continue
        d.append(max(abs(v["tmq"] - w["tmq"]), abs(v["tmr"] - w["tmr"])))
        same.append(v["query_aln"] == w["query_aln"] and v["refrn_aln"] == w["refrn_aln"])
    d = np.array(d)
    return {"pairs": len(d), "frac_tm_1e4": float((d <= 1e-4).mean()) if len(d) else 1.0,
            "frac_aln_identical": float(np.mean(same)) if same else 1.0}


def main():
    import argparse
    ap = argparse.ArgumentParser()
    ap.add_argument("sets", nargs="*")
    ap.add_argument("--gpu", action="store_true", help="run the reference's GPU build")
    ap.add_argument("--outdir", default=HERE)
    a = ap.parse_args()
    binary = BIN_GPU if a.gpu else BIN
    if not os.path.exists(binary):
        sys.exit("build the reference first: make -f oracle/Makefile.ref%s" % ("gpu" if a.gpu else ""))
    names = a.sets or list(SETS)
    for name in names:
        mk, opts = SETS[name][:2]
        threads = SETS[name][2] if len(SETS[name]) > 2 else 8
        runf = run_perpair if len(SETS[name]) > 3 and SETS[name][3] == "perpair" else run
        wl = mk()
        res = runf(wl, opts, threads, binary)
        wl2 = copy.deepcopy(wl)
        rng = np.random.default_rng(7)
        R = synth._rot_random(rng)
        q = wl2.queries[0]
        q.xyz = synth._pdb_round_fast(q.xyz.astype(np.float64) @ R.T + np.array([3.0, -5.0, 7.0]))
        res2 = runf(wl2, opts, threads, binary)
        if a.gpu:
            out = {"options": opts, "seed_desc": wl.desc, "results": res,
                   "self_agreement": agreement(res, res2), "binary": "reference GPU build (sm_100a)"}
            cpu = os.path.join(HERE, name + ".json")
            if os.path.exists(cpu):
                out["agreement_with_cpu_build"] = agreement(res, json.load(open(cpu))["results"])
            os.makedirs(a.outdir, exist_ok=True)
            with open(os.path.join(a.outdir, name + "_refgpu.json"), "w") as f:
                json.dump(out, f, indent=0, sort_keys=True)
            print(name, len(res), "pairs; GPU build self-agreement:", out["self_agreement"],
                  "vs CPU build:", out.get("agreement_with_cpu_build"))
            continue
        arrs = {}
        for tag, chains in (("q", wl.queries), ("r", wl.refs)):
            s = synth.pack(chains)
            arrs[tag + "_lens"] = s.lens
            arrs[tag + "_xyz"] = np.stack([s.x, s.y, s.z], axis=1)
            arrs[tag + "_rsd"] = s.rsd
            arrs[tag + "_mol"] = s.mol
            arrs[tag + "_names"] = np.array([c.name for c in chains])
        # sets on another set's inputs (the same builder) keep one input file
        if name not in ("c0_full_s13",):
            np.savez_compressed(os.path.join(a.outdir, name + ".npz"), **arrs)
        with open(os.path.join(a.outdir, name + ".json"), "w") as f:
            json.dump({"options": opts, "seed_desc": wl.desc, "results": res,
                       "self_agreement": agreement(res, res2)}, f, indent=0, sort_keys=True)
        print(name, len(res), "pairs; reference self-agreement:", agreement(res, res2))


if __name__ == "__main__":
    main()
