"""Loading of the golden fixtures made by tests/golden/make_golden.py."""
import json
import os

import numpy as np

from gtalign_alpha_b200.synth import SoA

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
# --refinement code -> the fixture set run at that code (homologs only)
LEVEL_SETS = {-1: "c0_level_m1", 0: "c0_level_0", 1: "c0_level_1", 2: "c0_level_2",
              3: "c0_level_3"}
SETS = ["c0_speed13", "c0_default", "c0_filters", "c0_sym_ref_nodel", "c0_shallow", "c0_2tm",
        "c0_ssrr", "c0_presim", "c0_na", "c0_combo"] + \
    list(LEVEL_SETS.values()) + ["c0_full", "c0_full_s13", "f3_default", "f3_speed12", "f3_opts",
                                 "f3_speed6", "f3_speed3", "f3_speed0"]
# the sets the GPU golden test runs: every set the CUDA library takes (it
# refuses nucleic-acid pairs) except the combined-options set, which pins
# the oracle only (each of its options runs on the GPU in the option sets)
LIBRARY_SETS = [s for s in SETS if s not in ("c0_na", "c0_combo", "c0_full", "c0_full_s13")]
# the small configuration at full size (1 x 1,000 pairs): default options
# without the detailed search, and --speed=13, on the same inputs
FULL_SETS = ["c0_full", "c0_full_s13"]
# sets whose inputs are another set's
INPUTS = {"c0_full_s13": "c0_full"}


def _soa(z, tag):
    lens = z[tag + "_lens"].astype(np.int32)
    offs = np.zeros_like(lens)
    if len(lens) > 1:
        offs[1:] = np.cumsum(lens[:-1])
    xyz = z[tag + "_xyz"].astype(np.float32)
    mol = z[tag + "_mol"].astype(np.int32) if tag + "_mol" in z else np.zeros(len(lens), np.int32)
    return SoA(lens, offs, np.ascontiguousarray(xyz[:, 0]), np.ascontiguousarray(xyz[:, 1]),
               np.ascontiguousarray(xyz[:, 2]), z[tag + "_rsd"].astype(np.uint8), mol)


def load(name):
    z = np.load(os.path.join(GOLDEN, INPUTS.get(name, name) + ".npz"))
    with open(os.path.join(GOLDEN, name + ".json")) as f:
        meta = json.load(f)
    return (_soa(z, "q"), _soa(z, "r"), list(z["q_names"]), list(z["r_names"]), meta)


def cli_options(opts):
    """Translate the reference CLI options of a set into oracle/library options."""
    d = dict(refinement=1, convergence=18, prescore=0.4, scorethld=0.5, depth=2,
             symmetric=0, referenced=0, nodeletions=0, twotmscore=0, addsearchbyss=0,
             presimilarity=0.0, nodetailedsearch=0 if "--no-detailed-search" not in opts else 1,
             trigger=50, seedrule=1, nbranches=5, gapcost=1, window=256)
    i = 0
    while i < len(opts):
        o = opts[i]
        if o == "--speed=13":
            d["refinement"], d["convergence"] = 0, 2
            d["nodetailedsearch"] = 1
        elif o.startswith("--refinement="):
            d["refinement"] = int(o.split("=")[1])
        elif o.startswith("--depth="):
            d["depth"] = int(o.split("=")[1])
        elif o.startswith("--convergence="):
            d["convergence"] = int(o.split("=")[1])
        elif o.startswith("--pre-score="):
            d["prescore"] = float(o.split("=")[1])
        elif o == "-s":
            d["scorethld"] = float(opts[i + 1]); i += 1
        elif o == "--symmetric":
            d["symmetric"] = 1
        elif o == "--referenced":
            d["referenced"] = 1
        elif o == "--no-deletions":
            d["nodeletions"] = 1
        elif o == "--2tm-score":
            d["twotmscore"] = 1
        elif o == "--add-search-by-ss":
            d["addsearchbyss"] = 1
        elif o.startswith("--pre-similarity="):
            d["presimilarity"] = float(o.split("=")[1])
        elif o.startswith("--speed="):
            sp = int(o.split("=")[1])
            d["nodetailedsearch"] = 0
            d["depth"] = 3 if sp >= 10 else (2 if sp >= 7 else (1 if sp >= 4 else 0))
            d["trigger"] = (0, 20, 50)[(sp - 1) % 3] if 1 <= sp <= 12 else 0
            if sp >= 10:
                d["refinement"], d["convergence"] = 0, 2
            if sp == 0:
                d["nbranches"], d["addsearchbyss"] = 16, 1
        elif o.startswith("--trigger="):
            d["trigger"] = int(o.split("=")[1])
        elif o.startswith("--seedrule="):
            d["seedrule"] = int(o.split("=")[1])
        elif o.startswith("--nbranches="):
            d["nbranches"] = int(o.split("=")[1])
        elif o.startswith("--gapcost="):
            d["gapcost"] = int(o.split("=")[1])
        elif o.startswith("--window="):
            d["window"] = int(o.split("=")[1])
        i += 1
    return d


def oracle_opts(oracle, d, cls=None):
    """oracle options from a cli_options dict (cls: a clustering run's
    prefilter, as pyoracle.opts_from takes it)"""
    return oracle.opts_from(cls=cls,
        refinement=d["refinement"], convergence=d["convergence"], prescore=d["prescore"],
        scorethld=d["scorethld"], symmetric=d["symmetric"], referenced=d["referenced"],
        nodeletions=d["nodeletions"], depth=d["depth"], twotmscore=d["twotmscore"],
        addsearchbyss=d["addsearchbyss"], presimilarity=d["presimilarity"],
        nodetailedsearch=d.get("nodetailedsearch", 1), trigger=d.get("trigger", 50),
        nbranches=d.get("nbranches", 5), gapcost=d.get("gapcost", 1),
        seedrule=d.get("seedrule", 1), window=d.get("window", 256))
