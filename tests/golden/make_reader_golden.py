"""Reader fixtures from the reference's CPU build: the structures it reads
from a set of crafted PDB files under each interpretation option set.

write_cases(dir) writes the files (seeded; the test rebuilds them the same
way).  For every option set the reference is run with the files as both
queries and references (-s 0, every hit reported); a structure's self-hit is
a gapless full-length alignment, so its query description, length and
aligned query sequence are what the reader made of it.  Stored in
tests/golden/reader_cases.json with the descriptions made relative to the
files' directory:

    python tests/golden/make_reader_golden.py
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
sys.path.insert(0, ROOT)
from gtalign_alpha_b200 import synth  # noqa: E402

BIN = os.path.join(ROOT, "oracle", "_ref", "gtalign")

OPTSETS = {
    "default": [],
    "hetatm": ["--hetatm"],
    "ter0": ["--ter=0"],
    "ter1": ["--ter=1"],
    "ter2": ["--ter=2"],
    "split1": ["--split=1", "--ter=0"],
    "split2": ["--split=2", "--ter=0"],
    "split2ter1": ["--split=2", "--ter=1"],
    "ter0max100": ["--ter=0", "--dev-max-length=100"],
    "aatom_n": ["--aatom= N  "],
    "infmt_pdb": ["--infmt=1"],
    "infmt_cif": ["--infmt=2"],
}

AA3 = ["ALA", "ARG", "ASN", "ASP", "CYS", "GLN", "GLU", "GLY", "HIS", "ILE", "LEU", "LYS",
       "MET", "PHE", "PRO", "SER", "THR", "TRP", "TYR", "VAL"]


def atom(rec, serial, name, alt, res, chain, num, icode, xyz):
    """One PDB coordinate record, 80 columns."""
    return ("%-6s%5d %-4s%1s%3s %1s%4d%1s   %8.3f%8.3f%8.3f  1.00  0.00           C  \n"
            % (rec, serial % 100000, name, alt, res, chain, num % 10000, icode,
               xyz[0], xyz[1], xyz[2]))


def chain_lines(rng, n, chain, start=1, rec_of=None, alts=None, icodes=None, names=None,
                extra_atoms=False, atomname=" CA "):
    """Records of an n-residue chain (C-alpha positions from the generator)."""
    c = synth.random_chains(rng, [n], "c")[0]
    out = []
    for i in range(n):
        res = names[i] if names else AA3[int(rng.integers(0, 20))]
        rec = rec_of(i) if rec_of else "ATOM"
        ic = icodes[i] if icodes else " "
        num = start + i
        if extra_atoms:
            out.append(atom(rec, 1, " N  ", " ", res, chain, num, ic, c.xyz[i] + 1.2))
        for alt in (alts(i) if alts else [" "]):
            shift = 0.0 if alt in " A" else 0.4
            out.append(atom(rec, 1, atomname, alt, res, chain, num, ic, c.xyz[i] + shift))
        if extra_atoms:
            out.append(atom(rec, 1, " C  ", " ", res, chain, num, ic, c.xyz[i] - 1.1))
            out.append(atom(rec, 1, " O  ", " ", res, chain, num, ic, c.xyz[i] - 2.0))
    return out


CIF_COLS = ["group_PDB", "id", "type_symbol", "label_atom_id", "label_alt_id", "label_comp_id",
            "label_asym_id", "label_entity_id", "label_seq_id", "pdbx_PDB_ins_code", "Cartn_x",
            "Cartn_y", "Cartn_z", "occupancy", "B_iso_or_equiv", "auth_seq_id", "auth_asym_id",
            "pdbx_PDB_model_num"]


def cif_file(rows, cols=CIF_COLS, pad=1):
    """A PDBx/mmCIF text with one _atom_site loop; rows are dicts of column
    values ('.' where absent); `pad` spaces between tokens."""
    out = ["data_TEST\n", "#\n", "_entry.id TEST\n", "#\n", "loop_\n"]
    out += ["_atom_site.%s \n" % c for c in cols]
    for r in rows:
        out.append((" " * pad).join(str(r.get(c, ".")) for c in cols) + "\n")
    out.append("#\n")
    return out


def cif_chain(rng, n, label_asym, auth_asym, model=1, seq0=1, rec_of=None, alts=None,
              icodes=None, names=None, atomname="CA", extra_atoms=False):
    c = synth.random_chains(rng, [n], "c")[0]
    rows = []
    for i in range(n):
        res = names[i] if names else AA3[int(rng.integers(0, 20))]
        base = {"group_PDB": rec_of(i) if rec_of else "ATOM", "type_symbol": "C",
                "label_comp_id": res, "label_asym_id": label_asym, "label_entity_id": 1,
                "label_seq_id": seq0 + i, "pdbx_PDB_ins_code": icodes[i] if icodes else "?",
                "occupancy": "1.00", "B_iso_or_equiv": "0.00", "auth_seq_id": seq0 + i,
                "auth_asym_id": auth_asym, "pdbx_PDB_model_num": model}
        if extra_atoms:
            rows.append(dict(base, label_atom_id="N", label_alt_id=".",
                             Cartn_x="%.3f" % (c.xyz[i][0] + 1), Cartn_y="%.3f" % c.xyz[i][1],
                             Cartn_z="%.3f" % c.xyz[i][2]))
        for alt in (alts(i) if alts else ["."]):
            sh = 0.0 if alt in ".A" else 0.4
            rows.append(dict(base, label_atom_id=atomname, label_alt_id=alt,
                             Cartn_x="%.3f" % (c.xyz[i][0] + sh), Cartn_y="%.3f" % c.xyz[i][1],
                             Cartn_z="%.3f" % c.xyz[i][2]))
    return rows


def _gz(b: bytes) -> bytes:
    import gzip
    return gzip.compress(b, mtime=0)


def ter_line(full=True):
    return "TER     999      ALA A 999                                                      \n" if full else "TER\n"


def write_cases(d: str) -> list:
    """Write the crafted files into d; returns their names in order."""
    rng = np.random.default_rng(101)
    files = {}
    files["a_plain.pdb"] = chain_lines(rng, 80, "A", extra_atoms=True) + ["END\n"]
    files["b_two_chains_ter.pdb"] = (chain_lines(rng, 50, "A") + [ter_line()] +
                                    chain_lines(rng, 40, "B") + [ter_line(), "END\n"])
    files["c_two_chains.pdb"] = chain_lines(rng, 45, "A") + chain_lines(rng, 35, "B") + ["END\n"]
    files["d_models.pdb"] = (["MODEL        1                                                                  \n"] +
                             chain_lines(rng, 60, "A") + ["ENDMDL\n",
                             "MODEL        2                                                                  \n"] +
                             chain_lines(rng, 55, "A") + ["ENDMDL\n", "END\n"])
    files["e_altloc.pdb"] = chain_lines(
        rng, 70, "A", alts=lambda i: ["A", "B"] if 10 <= i < 15 else (["C"] if i == 20 else [" "])) + ["END\n"]
    files["f_hetatm.pdb"] = chain_lines(
        rng, 60, "A", rec_of=lambda i: "HETATM" if 20 <= i < 26 else "ATOM",
        names=[("MSE" if 20 <= i < 26 else AA3[i % 20]) for i in range(60)]) + ["END\n"]
    files["g_short_first.pdb"] = chain_lines(rng, 10, "A") + chain_lines(rng, 50, "B") + ["END\n"]
    files["h_icodes.pdb"] = chain_lines(
        rng, 40, "A", start=45, icodes=[("A" if i % 7 == 3 else " ") for i in range(40)]) + ["END\n"]
    files["i_rna_protein.pdb"] = (chain_lines(rng, 40, "A", atomname=" C3'",
                                              names=["  " + "ACGU"[i % 4] for i in range(40)]) +
                                  [ter_line()] + chain_lines(rng, 30, "B") + ["END\n"])
    files["j_unknown_names.pdb"] = chain_lines(
        rng, 30, "A", names=[("UNK" if i % 5 == 0 else (" DA" if i % 5 == 1 else AA3[i % 20]))
                             for i in range(30)]) + ["END\n"]
    files["k_short_lines.pdb"] = (chain_lines(rng, 40, "A") + [ter_line(False)] +
                                  chain_lines(rng, 45, "B") + ["END\n"])
    files["l_blank_chain.pdb"] = chain_lines(rng, 40, " ") + ["END\n"]
    for n in (100, 101, 102):                # around --dev-max-length=100
        files["m_len%d.pdb" % n] = chain_lines(rng, n, "A") + ["END\n"]
    # PDBx/mmCIF
    files["n_cif_plain.cif"] = cif_file(cif_chain(rng, 70, "A", "A", extra_atoms=True))
    files["o_cif_two_chains.cif"] = cif_file(cif_chain(rng, 50, "A", "X") + cif_chain(rng, 40, "B", "Y"))
    files["p_cif_models.cif"] = cif_file(cif_chain(rng, 45, "A", "A", model=1) +
                                         cif_chain(rng, 45, "A", "A", model=2))
    files["q_cif_altloc_hetatm.cif"] = cif_file(cif_chain(
        rng, 60, "A", "A", alts=lambda i: ["A", "B"] if 5 <= i < 9 else (["C"] if i == 12 else ["."]),
        rec_of=lambda i: "HETATM" if 30 <= i < 34 else "ATOM",
        names=[("MSE" if 30 <= i < 34 else ("DAL" if i == 40 else AA3[i % 20])) for i in range(60)]))
    files["r_cif_rna.cif"] = cif_file(cif_chain(rng, 40, "A", "A", atomname='"C3\'"',
                                                names=["ACGU"[i % 4] for i in range(40)]))
    files["s_cif_icodes_label_only.cif"] = cif_file(
        cif_chain(rng, 35, "A", "A", icodes=[("B" if i % 6 == 2 else "?") for i in range(35)]),
        cols=[c for c in CIF_COLS if not c.startswith("auth_")])
    # tokens past a record's 128th character are not read: with wide spacing
    # the chain, number and model come from the label columns or not at all
    files["t_cif_wide.cif"] = cif_file(cif_chain(rng, 30, "A", "Z", model=3), pad=7)
    files["u_cif.gz"] = cif_file(cif_chain(rng, 25, "A", "A"))     # .gz without .cif: read as PDB
    # a tar archive: a PDB, a PDBx/mmCIF and a gzip-compressed PDB entry, a
    # directory entry and a file under 10 bytes
    tar_entries = [("t1.pdb", "".join(chain_lines(rng, 33, "A") + ["END\n"]).encode()),
                   ("sub/t2.cif", "".join(cif_file(cif_chain(rng, 28, "B", "B"))).encode()),
                   ("t3.pdb.gz", _gz("".join(chain_lines(rng, 41, "C") + ["END\n"]).encode())),
                   ("tiny.pdb", b"END\n")]
    import io
    import tarfile
    with tarfile.open(os.path.join(d, "v_archive.tar"), "w", format=tarfile.USTAR_FORMAT) as t:
        di = tarfile.TarInfo("sub")
        di.type = tarfile.DIRTYPE
        di.mtime = 0
        t.addfile(di)
        for name, data in tar_entries:
            ti = tarfile.TarInfo(name)
            ti.size = len(data)
            ti.mtime = 0
            t.addfile(ti, io.BytesIO(data))
    for name, lines in files.items():
        if name.endswith(".gz"):
            import gzip
            with gzip.open(os.path.join(d, name), "wt") as f:
                f.writelines(lines)
            continue
        with open(os.path.join(d, name), "w") as f:
            f.writelines(lines)
    return sorted(list(files) + ["v_archive.tar"])


def run_reference(d: str, opts: list) -> list:
    """[(description relative to d, length, sequence)] of the structures the
    reference reads as references (those with a self-hit; the query side has
    its own length limit), sorted by description."""
    with tempfile.TemporaryDirectory(prefix="gtrd") as out:
        r = subprocess.run([BIN, "--qrs=" + d, "--rfs=" + d, "-o", out, "--outfmt=1", "-s", "0",
                            "--no-detailed-search", "--cpu-threads=8"] + opts,
                           capture_output=True, text=True, timeout=600)
        if r.returncode != 0:
            raise RuntimeError(r.stderr[-2000:])
        rec = []
        for f in os.listdir(out):
            J = json.load(open(os.path.join(out, f)))["gtalign_search"]
            qd, ql = J["query"]["description"], J["query"]["length"]
            seq = None
            for h in J["search_results"]:
                h = h["hit_record"]
                if h["reference_description"] == qd:
                    a = h["alignment"]
                    if a["n_aligned"] == ql and a["query_from"] == 1 and a["query_to"] == ql:
                        seq = a["query_aln"]
            if seq is not None:
                rec.append((os.path.relpath(qd, d) if qd.startswith(d) else qd, ql, seq))
    return sorted(rec)


def main():
    res = {}
    with tempfile.TemporaryDirectory(prefix="gtrdc") as d:
        names = write_cases(d)
        for key, opts in OPTSETS.items():
            res[key] = {"options": opts, "structures": run_reference(d, opts)}
            print(key, len(res[key]["structures"]), "structures")
    out = {"files": names, "sets": res, "generator": "tests/golden/make_reader_golden.py"}
    with open(os.path.join(HERE, "reader_cases.json"), "w") as f:
        json.dump(out, f, indent=1)


if __name__ == "__main__":
    main()
