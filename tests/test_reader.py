"""The host reader (gtb_read_pdb) against the reference's own reader.

tests/golden/reader_cases.json holds, for each interpretation option set,
the structures the reference's CPU build read from a set of crafted PDB
files (description, length, sequence; tests/golden/make_reader_golden.py):
chains split or joined by TER / END / ENDMDL / chain changes, models,
alternate locations, HETATM residues, insertion codes, a nucleic-acid
chain, unknown residue names, a chain below the minimum length, short
records, lengths around --dev-max-length; PDBx/mmCIF files; a tar archive
with plain, mmCIF and gzip entries.  The reader must yield exactly those
structures.  Host code: no device needed.
"""
import gzip
import json
import os
import shutil
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))

FIX = os.path.join(HERE, "golden", "reader_cases.json")


def _opts(flags):
    kw = {}
    for f in flags:
        if f == "--hetatm":
            kw["hetatm"] = True
        elif f.startswith("--dev-max-length="):
            kw["maxlen"] = int(f.split("=")[1])
        elif f.startswith("--aatom="):
            kw["aatom"] = f[len("--aatom="):]
        else:
            k, v = f[2:].split("=")
            kw[k] = int(v)
    return kw


@pytest.fixture(scope="module")
def cases(tmp_path_factory):
    import make_reader_golden as mrg
    d = str(tmp_path_factory.mktemp("reader"))
    names = mrg.write_cases(d)
    return d, names


@pytest.mark.parametrize("key", ["default", "hetatm", "ter0", "ter1", "ter2", "split1", "split2",
                                 "split2ter1", "ter0max100", "aatom_n", "infmt_pdb",
                                 "infmt_cif"])
def test_reader_reads_what_the_reference_reads(cases, key):
    from gtalign_alpha_b200.api import read_pdb
    fx = json.load(open(FIX))
    d, names = cases
    assert names == fx["files"]
    rb = read_pdb([os.path.join(d, n) for n in names], threads=3, **_opts(fx["sets"][key]["options"]))
    s = rb.soa
    ours = []
    for i, desc in enumerate(rb.descriptions):
        o, n = int(s.offs[i]), int(s.lens[i])
        seq = bytes(s.rsd[o:o + n]).decode()
        ours.append([os.path.relpath(desc, d), n, seq])
    assert sorted(ours) == sorted([list(t) for t in fx["sets"][key]["structures"]])


def test_reader_round_trip_and_layout(tmp_path):
    """Chains written by synth.write_pdb (one file each, one gzip-compressed)
    come back with their coordinates (to the file's 3 decimals), residue
    letters, lengths and offsets; the packed fields have the reference's
    layout (per-residue insertion/chain/order value negated for protein)."""
    from gtalign_alpha_b200 import synth
    from gtalign_alpha_b200.api import read_pdb
    rng = np.random.default_rng(5)
    chains = synth.random_chains(rng, [35, 120, 60, 250], "r")
    paths = []
    for k, c in enumerate(chains):
        p = str(tmp_path / ("s%d.pdb" % k))
        synth.write_pdb(c, p)
        if k == 1:
            with open(p, "rb") as f, gzip.open(p + ".gz", "wb") as g:
                shutil.copyfileobj(f, g)
            p += ".gz"
        paths.append(p)
    for threads in (1, 4):
        rb = read_pdb(paths, threads=threads)
        s = rb.soa
        assert s.n == 4 and list(s.lens) == [c.length for c in chains]
        assert list(s.offs) == list(np.cumsum([0] + [c.length for c in chains])[:-1])
        xyz = np.stack([s.x, s.y, s.z], 1)
        ref = np.concatenate([c.xyz for c in chains]).astype(np.float32)
        assert np.abs(xyz - np.round(ref.astype(np.float64), 3)).max() < 1e-4
        assert bytes(s.rsd).decode() == "".join(bytes(c.seq).decode() for c in chains)
        assert (s.mol == 0).all()
        pk = rb.packed
        assert pk.n == 4 and pk.npos == s.total
        insch = pk.arrays[6]
        assert (insch < 0).all()                      # protein residues
        assert ((-insch >> 8) & 0xff == ord("A")).all() and ((-insch) & 0xff == 1).all()
        assert rb.descriptions[0] == paths[0] + " Chn:A"


def test_reader_errors(tmp_path):
    from gtalign_alpha_b200.api import GTBError, read_pdb
    p = tmp_path / "x.cif"
    p.write_text("data_1ABC\nloop_\n_atom_site.group_PDB\n")
    assert read_pdb([str(p)]).soa.n == 0                  # no complete atom table
    t = tmp_path / "x.tar"
    t.write_bytes(b"0" * 1024)                            # a bad checksum: nothing listed
    assert read_pdb([str(t)]).soa.n == 0
    with pytest.raises(GTBError) as e:
        read_pdb([str(tmp_path / "nope.pdb")])
    assert e.value.status == 1
    with pytest.raises(GTBError):
        read_pdb([str(p)], ter=7)
    for bad in (dict(split=1, ter=1), dict(split=2, ter=2), dict(split=2)):   # the CLI's rules
        with pytest.raises(GTBError):
            read_pdb([str(p)], **bad)


def test_reader_length_limits(tmp_path):
    """--dev-min-length drops shorter structures; --dev-max-length drops a
    structure once more residues than the limit are stored before the next
    one (the reference's comparison, which admits one residue above it)."""
    from gtalign_alpha_b200 import synth
    from gtalign_alpha_b200.api import read_pdb
    rng = np.random.default_rng(6)
    paths = []
    for k, n in enumerate((19, 20, 100, 101, 102)):
        c = synth.random_chains(rng, [n], "m")[0]
        paths.append(str(tmp_path / ("m%d.pdb" % k)))
        synth.write_pdb(c, paths[-1])
    rb = read_pdb(paths, maxlen=100)
    assert list(rb.soa.lens) == [20, 100, 101]


def test_coordinate_parser_equals_strtof(tmp_path):
    """The reader's fast decimal path gives strtof's float for every
    coordinate a PDB record can hold (-999.999 .. 9999.999 in steps of
    0.001, the "%8.3f" field) and for random decimals of up to 6 places and
    9 digits, and its integer path strtol's value for every "%4d" residue
    number and a few odd fields (compiled with the host compiler around the
    reader's source)."""
    import subprocess
    src = tmp_path / "fp.cpp"
    src.write_text(r'''
#include "%s"
#include <random>
int main() {
    char buf[32];
    long bad = 0, n = 0;
    for (long m = -999999; m <= 9999999; m++) {
        std::snprintf(buf, sizeof buf, "%%8.3f", m / 1000.0);
        float a = 0.f, b = std::strtof(buf, nullptr);
        if (!field_float(buf, 8, a) || std::memcmp(&a, &b, 4) != 0) bad++;
        n++;
    }
    std::mt19937_64 g(7);
    for (int k = 0; k < 3000000; k++) {
        int d = (int)(g() %% 7), nd = 1 + (int)(g() %% 9);
        if (d > nd) d = nd;
        long long m = (long long)(g() %% 1000000000ULL);
        long long lim = 1; for (int i = 0; i < nd; i++) lim *= 10;
        m %%= lim;
        char digits[16];
        std::snprintf(digits, sizeof digits, "%%0*lld", nd, m);
        std::string s = (g() & 1) ? "-" : " ";
        s += std::string(digits, (size_t)(nd - d));
        if (d) s += "." + std::string(digits + nd - d, (size_t)d);
        float a = 0.f, b = std::strtof(s.c_str(), nullptr);
        if (!field_float(s.c_str(), (int)s.size(), a) || std::memcmp(&a, &b, 4) != 0) bad++;
        n++;
    }
    for (long m = -999; m <= 9999; m++) {                 // the "%%4d" residue number field
        std::snprintf(buf, sizeof buf, "%%4ld", m);
        int a = 0;
        long b = std::strtol(buf, nullptr, 10);
        if (!field_int(buf, 4, a) || a != (int)b) bad++;
        n++;
    }
    for (const char* t : {"  1A", " -0 ", "+12 ", "    ", " x12", "1234", "\t 7\t"}) {
        int a = 0;
        char* e = nullptr;
        long b = std::strtol(t, &e, 10);
        const bool ok = field_int(t, 4, a);
        if (ok != (e != t) || (ok && a != (int)b)) bad++;
        n++;
    }
    std::printf("%%ld %%ld\n", n, bad);
    return bad != 0;
}
''' % os.path.join(os.path.dirname(HERE), "gtalign_alpha_b200", "csrc", "gtb_reader.cpp"))
    exe = tmp_path / "fp"
    subprocess.check_call(["g++", "-O2", "-std=c++17", "-I", os.path.join(os.path.dirname(HERE), "include"),
                           "-o", str(exe), str(src), "-lz", "-lpthread"])
    out = subprocess.run([str(exe)], capture_output=True, text=True)
    n, bad = (int(x) for x in out.stdout.split())
    assert n > 13_000_000 and bad == 0, out.stdout


def test_reader_survives_truncated_and_garbage_files(cases, tmp_path):
    """Every crafted file cut at random offsets, and random bytes under each
    file name form, read without a crash (structures or a status code)."""
    from gtalign_alpha_b200.api import GTBError, read_pdb
    d, names = cases
    rng = np.random.default_rng(17)
    paths = []
    for k in range(120):
        src = os.path.join(d, names[k % len(names)])
        data = open(src, "rb").read()
        cut = int(rng.integers(0, len(data) + 1))
        ext = os.path.splitext(names[k % len(names)])[1]
        p = str(tmp_path / ("cut%03d%s" % (k, ext)))
        with open(p, "wb") as f:
            f.write(data[:cut])
        paths.append(p)
    for k, ext in enumerate([".pdb", ".cif", ".gz", ".tar", ".ent"] * 6):
        p = str(tmp_path / ("rnd%03d%s" % (k, ext)))
        with open(p, "wb") as f:
            f.write(rng.integers(0, 256, int(rng.integers(0, 3000)), dtype=np.uint8).tobytes())
        paths.append(p)
    ok = 0
    for p in paths:
        try:
            read_pdb([p])
            ok += 1
        except GTBError:
            pass
    assert ok > 60
