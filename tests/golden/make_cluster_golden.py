"""Clustering fixtures from the reference's GPU build (its --cls mode).

The reference clusters only in its GPU build ("The clustering option is
available only in the GPU version"): oracle/_ref/gpu/gtalign, compiled for
sm_100a from the reference sources by oracle/Makefile.refgpu.  This script
writes a seeded set of structure families as PDB files, runs

    gtalign --cls=<file>,<file>,... -o <out> --speed=13 --cls-threshold=T --cls-algorithm=A

and stores the clusters it lists in gtalignclusters.lst (a line per cluster,
the representative first) as tests/golden/cls_<name>.json, together with
the generator's parameters (the test rebuilds the structures from them).
Run it on a machine with a GPU:

    python tests/golden/make_cluster_golden.py [--outdir DIR]
"""
from __future__ import annotations

import argparse
import json
import os
import re
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
from gtalign_alpha_b200 import synth  # noqa: E402

BIN_GPU = os.path.join(ROOT, "oracle", "_ref", "gpu", "gtalign")
NAME = re.compile(r"clsf\d\dm\d\d")

# name -> (seed, families, members, noise sigma, indel fraction, linkage, threshold)
SETS = {
    "cls_complete": dict(seed=51, families=8, members=5, sigma=0.9, indel=0.04, linkage=0, threshold=0.5),
    "cls_single": dict(seed=52, families=6, members=6, sigma=1.2, indel=0.06, linkage=1, threshold=0.5),
    # members drawn from 1.0 to 3.0 A of noise, so that some fall near or out
    # of the threshold
    "cls_mixed_single": dict(seed=53, families=6, members=5, sigma=1.0, sigma_hi=3.0, indel=0.05,
                             linkage=1, threshold=0.5),
}


def structures(p):
    """The set: `families` unrelated chains of 70-220 residues, each with
    `members` - 1 noisy, indel-bearing, moved copies; names clsfFFmMM
    (member 0 the family's first chain)."""
    rng = np.random.default_rng(p["seed"])
    lens = [int(x) for x in rng.integers(70, 220, size=p["families"])]
    base = synth.random_chains(rng, lens, "b")
    out = []
    for f, b in enumerate(base):
        out.append(synth.Chain(b.xyz, b.seq, "clsf%02dm%02d" % (f, 0)))
        for m in range(1, p["members"]):
            sigma = p["sigma"]
            if "sigma_hi" in p:
                sigma = float(rng.uniform(p["sigma"], p["sigma_hi"]))
            h = synth.homolog(rng, b, sigma, p["indel"], "clsf%02dm%02d" % (f, m))
            out.append(h)
    return out


def run_reference(p, chains, workdir):
    sdir = os.path.join(workdir, "s")
    odir = os.path.join(workdir, "o")
    os.makedirs(sdir, exist_ok=True)
    files = []
    for c in sorted(chains, key=lambda c: c.name):
        files.append(os.path.join(sdir, c.name + ".pdb"))
        synth.write_pdb(c, files[-1])
    # the structures as a list of files, in name order: the reader numbers
    # them (their global indices, the clustering order) in that order
    cmd = [BIN_GPU, "--cls=" + ",".join(files), "-o", odir, "--speed=13", "--dev-N=1",
           "--cls-threshold=%g" % p["threshold"], "--cls-algorithm=%d" % p["linkage"]]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=600)
    if r.returncode != 0:
        raise RuntimeError("reference --cls run failed: %s" % r.stderr[-2000:])
    clusters = []
    with open(os.path.join(odir, "gtalignclusters.lst")) as f:
        text = f.read()
    lines = text.splitlines()
    # the cluster lines follow the last rule of '=' under the header (which
    # lists the command line and the structures clustered)
    last = max(k for k, ln in enumerate(lines) if ln.startswith("===="))
    for line in lines[last + 1:]:
        names = []
        for nm in NAME.findall(line):      # a name may occur in a member's path and id
            if nm not in names:
                names.append(nm)
        if names:
            clusters.append(names)
    return clusters, " ".join(cmd[1:]), text


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--outdir", default=HERE)
    ap.add_argument("sets", nargs="*")
    a = ap.parse_args()
    for name in a.sets or list(SETS):
        p = SETS[name]
        chains = structures(p)
        with tempfile.TemporaryDirectory(prefix="gtcls") as wd:
            clusters, cmd, text = run_reference(p, chains, wd)
        seen = sorted(n for c in clusters for n in c)
        if seen != sorted(c.name for c in chains):
            with open(os.path.join(a.outdir, name + ".lst"), "w") as f:
                f.write(text)
            raise RuntimeError("%s: the clusters do not list every structure once" % name)
        cmd = cmd.replace(os.path.dirname(cmd.split("--cls=")[1].split(",")[0]) + "/", "")
        rec = {"params": p, "command": cmd, "clusters": clusters,
               "generator": "tests/golden/make_cluster_golden.py"}
        with open(os.path.join(a.outdir, name + ".json"), "w") as f:
            json.dump(rec, f, indent=1)
        print(name, len(clusters), "clusters")


if __name__ == "__main__":
    main()
