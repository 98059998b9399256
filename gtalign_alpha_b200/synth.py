"""Seeded synthetic C-alpha traces for the superposition-search workloads.

No public dataset is used anywhere in this package.  Chains are built with the
NeRF (natural extension reference frame) construction from virtual-bond
internal coordinates:

* every C-alpha to C-alpha virtual bond is 3.8 A long;
* coil residues draw the virtual bond angle from N(105 deg, 10 deg) and the
  torsion uniformly;
* helix runs use a bond angle of 91 deg and a torsion of 50 deg, which gives
  a rise of 1.5 A and 100 deg per residue;
* strand runs use a bond angle of 120 deg and a torsion of -170 deg, which
  gives a rise of about 3.3 A per residue;
* helix and strand runs are 4-20 residues long.

Homologs are copies of a template with 0..max indel fraction of random
insertions/deletions, Gaussian coordinate noise of a chosen sigma, and a random
rigid rotation and translation.

Coordinates are rounded to the 3 decimals a PDB ATOM record carries and are
converted to float32 the way ``std::stof`` does (``strtof``), so the arrays
handed to the C-ABI and the PDB files read by the reference hold the same
values.
"""
from __future__ import annotations

import ctypes
import math
import os
from dataclasses import dataclass, field
from typing import List, Optional, Sequence, Tuple

import numpy as np

AA = np.frombuffer(b"ACDEFGHIKLMNPQRSTVWY", dtype=np.uint8)
AA3 = {
    "A": "ALA", "C": "CYS", "D": "ASP", "E": "GLU", "F": "PHE", "G": "GLY",
    "H": "HIS", "I": "ILE", "K": "LYS", "L": "LEU", "M": "MET", "N": "ASN",
    "P": "PRO", "Q": "GLN", "R": "ARG", "S": "SER", "T": "THR", "V": "VAL",
    "W": "TRP", "Y": "TYR",
}

_libc = ctypes.CDLL(None)
_libc.strtof.restype = ctypes.c_float
_libc.strtof.argtypes = [ctypes.c_char_p, ctypes.c_void_p]


@dataclass
class Chain:
    """One structure: float32 SoA coordinates, residue letters, a name."""
    xyz: np.ndarray            # (L, 3) float32
    seq: np.ndarray            # (L,) uint8 residue letters
    name: str = "chain"
    na: bool = False           # nucleic acid: C3' atoms, bases A/C/G/U

    @property
    def length(self) -> int:
        return int(self.xyz.shape[0])


def _rot_random(rng: np.random.Generator) -> np.ndarray:
    q = rng.normal(size=4)
    q /= np.linalg.norm(q)
    a, b, c, d = q
    return np.array([
        [a*a + b*b - c*c - d*d, 2*(b*c - a*d), 2*(b*d + a*c)],
        [2*(b*c + a*d), a*a - b*b + c*c - d*d, 2*(c*d - a*b)],
        [2*(b*d - a*c), 2*(c*d + a*b), a*a - b*b - c*c + d*d]])


def _internal_coords(rng: np.random.Generator, L: int):
    """Bond angles and torsions (radians) for a chain of L residues."""
    theta = np.deg2rad(rng.normal(105.0, 10.0, size=L))
    tau = rng.uniform(-np.pi, np.pi, size=L)
    nseg = L // 2 + 2
    kind = rng.random(nseg)
    seglen = np.where(kind < 0.6, rng.integers(4, 21, size=nseg), rng.integers(2, 9, size=nseg))
    per = np.repeat(kind, seglen)[:L]
    hel = per < 0.35
    strd = (per >= 0.35) & (per < 0.6)
    theta[hel] = np.deg2rad(91.0)
    tau[hel] = np.deg2rad(50.0)
    theta[strd] = np.deg2rad(120.0)
    tau[strd] = np.deg2rad(-170.0)
    return theta, tau


def _nerf_flat(theta: np.ndarray, tau: np.ndarray, lens: np.ndarray, bond: float = 3.8) -> np.ndarray:
    """NeRF for many chains at once.  Chains are sorted by decreasing length;
    theta/tau are flat arrays (chain k owns [off[k], off[k]+lens[k])).
    Returns flat (sum(lens), 3) coordinates."""
    n = len(lens)
    off = np.zeros(n, np.int64)
    off[1:] = np.cumsum(lens[:-1])
    out = np.zeros((int(lens.sum()), 3))
    Lmax = int(lens.max()) if n else 0
    # window of the last three atoms per chain
    a = np.zeros((n, 3)); b = np.zeros((n, 3)); c = np.zeros((n, 3))
    for i in range(Lmax):
        m = int(np.searchsorted(-lens, -i, side="left"))  # chains with lens > i are [0, m)
        m = int((lens > i).sum()) if m == 0 or lens[m - 1] <= i else m
        if m == 0:
            break
        idx = off[:m] + i
        if i == 0:
            p = np.zeros((m, 3))
        elif i == 1:
            p = np.zeros((m, 3)); p[:, 0] = bond
        elif i == 2:
            t = theta[idx]
            p = np.zeros((m, 3)); p[:, 0] = bond - bond * np.cos(t); p[:, 1] = bond * np.sin(t)
        else:
            A, Bv, C = a[:m], b[:m], c[:m]
            bc = C - Bv
            bc /= np.linalg.norm(bc, axis=1, keepdims=True)
            nn = np.cross(Bv - A, bc)
            nl = np.linalg.norm(nn, axis=1, keepdims=True)
            nl[nl < 1e-9] = 1.0
            nn /= nl
            mm = np.cross(nn, bc)
            th, to = theta[idx], tau[idx]
            d0 = -bond * np.cos(th)
            d1 = bond * np.sin(th) * np.cos(to)
            d2 = bond * np.sin(th) * np.sin(to)
            p = C + d0[:, None] * bc + d1[:, None] * mm + d2[:, None] * nn
        out[idx] = p
        a[:m], b[:m], c[:m] = b[:m], c[:m], p
    return out


def _pdb_round_fast(x: np.ndarray) -> np.ndarray:
    """Round to 3 decimals and convert to float32 as strtof would.

    The 3-decimal value k/1000 is formed in float64 and rounded to float32.
    Double rounding (decimal -> float64 -> float32) can differ from a direct
    decimal -> float32 conversion only when the float64 value lies within
    2**-29 relative of a float32 rounding boundary; such values are converted
    again with strtof.
    """
    k = np.round(np.asarray(x, dtype=np.float64) * 1000.0)
    d = k / 1000.0
    f = d.astype(np.float32)
    back = f.astype(np.float64)
    ulp = np.abs(np.spacing(f).astype(np.float64))
    frac = np.abs(d - back) / ulp
    risky = np.abs(frac - 0.5) < 1e-6
    if np.any(risky):
        ff = f.ravel()
        dd = d.ravel()
        for i in np.nonzero(risky.ravel())[0]:
            ff[i] = _libc.strtof(("%.3f" % dd[i]).encode(), None)
        f = ff.reshape(f.shape)
    return f


def random_chains(rng: np.random.Generator, lengths: Sequence[int],
                  prefix: str = "rnd") -> List[Chain]:
    """Unrelated random-walk chains with helix/strand runs."""
    lengths = np.asarray([int(l) for l in lengths], dtype=np.int64)
    n = len(lengths)
    if n == 0:
        return []
    order = np.argsort(-lengths, kind="stable")
    sl = lengths[order]
    ths, tos = [], []
    for k in range(n):
        t1, t2 = _internal_coords(rng, int(sl[k]))
        ths.append(t1); tos.append(t2)
    X = _nerf_flat(np.concatenate(ths), np.concatenate(tos), sl)
    shifts = rng.uniform(-20, 20, size=(n, 3))
    seqs = AA[rng.integers(0, len(AA), size=int(sl.sum()))]
    out: List[Optional[Chain]] = [None] * n
    o = 0
    for j in range(n):
        L = int(sl[j])
        xyz = X[o:o + L]
        xyz = xyz - xyz.mean(axis=0) + shifts[j]
        k = int(order[j])
        out[k] = Chain(_pdb_round_fast(xyz), seqs[o:o + L].copy(), f"{prefix}{k:06d}")
        o += L
    return out  # type: ignore[return-value]


def homolog(rng: np.random.Generator, tmpl: Chain, sigma: float,
            indel_frac: float, name: str) -> Chain:
    """A noisy, indel-bearing, rigidly moved copy of ``tmpl``."""
    xyz = tmpl.xyz.astype(np.float64)
    seq = tmpl.seq
    L = xyz.shape[0]
    nindel = int(round(indel_frac * L))
    pos = rng.integers(0, L, size=nindel)
    isdel = rng.random(nindel) < 0.5
    keep = np.ones(L, dtype=bool)
    keep[pos[isdel]] = False
    nins = np.zeros(L, dtype=np.int64)
    np.add.at(nins, pos[~isdel], rng.integers(1, 4, size=int((~isdel).sum())))
    # each kept residue, then its insertions (random 3.8 A steps from it)
    reps = keep.astype(np.int64) + nins
    src = np.repeat(np.arange(L), reps)
    first = np.zeros(len(src), dtype=bool)
    starts = np.cumsum(reps) - reps
    kept_first = starts[keep & (reps > 0)]
    first[kept_first] = True
    P = xyz[src].copy()
    ins = ~first
    if ins.any():
        steps = rng.normal(size=(int(ins.sum()), 3))
        steps *= 3.8 / np.linalg.norm(steps, axis=1, keepdims=True)
        # cumulative walk within each insertion run
        run_id = np.cumsum(first)
        d = np.zeros_like(P)
        d[ins] = steps
        cs = np.cumsum(d, axis=0)
        base = np.zeros_like(P)
        idx_first = np.nonzero(first)[0]
        if len(idx_first):
            base = cs[idx_first][np.clip(run_id - 1, 0, len(idx_first) - 1)]
        P = P + (cs - base) * ins[:, None]
    aas = seq[src].copy()
    mut = (rng.random(len(src)) >= 0.6) | ins
    aas[mut] = AA[rng.integers(0, 20, size=int(mut.sum()))]
    P = P + rng.normal(0.0, sigma, size=P.shape)
    R = _rot_random(rng)
    P = (P - P.mean(axis=0)) @ R.T + rng.uniform(-30, 30, size=3)
    return Chain(_pdb_round_fast(P), aas.astype(np.uint8), name)


NA_COMPLEMENT = {"A": "U", "U": "A", "G": "C", "C": "G"}


def na_hairpins(rng: np.random.Generator, n_hairpins: int, stem: int, loop: int,
                name: str, noise: float = 0.3, rise: float = 5.9) -> Chain:
    """A nucleic-acid chain of C3' atoms: hairpins in a row, each an
    antiparallel stem of ``stem`` complementary base pairs whose C3' atoms
    are 13.75 A apart (the middle of the 12.5-15 A pairing window of the
    reference's base-pair assignment), ``rise`` A between stem neighbours,
    closed by a ``loop``-residue arc; hairpins 30 A apart, joined by 2
    residues."""
    pts, seq = [], []
    for h in range(n_hairpins):
        x0 = 30.0 * h
        s1 = [rng.choice(list("ACGU")) for _ in range(stem)]
        if h > 0:   # linker from the previous hairpin's last residue
            for t in (1, 2):
                pts.append((x0 - 16.25 + 5.4 * t, 0.0, -3.0))
                seq.append(rng.choice(list("ACGU")))
        for k in range(stem):
            pts.append((x0, 0.0, rise * k))
            seq.append(s1[k])
        top = rise * (stem - 1)
        for t in range(loop):
            a = np.pi * (t + 1) / (loop + 1)
            pts.append((x0 + 6.875 - 6.875 * np.cos(a), 2.0 * np.sin(a), top + 6.0 * np.sin(a)))
            seq.append(rng.choice(list("ACGU")))
        for k in range(stem - 1, -1, -1):
            pts.append((x0 + 13.75, 0.0, rise * k))
            seq.append(NA_COMPLEMENT[s1[k]])
    xyz = np.array(pts, dtype=np.float64) + rng.normal(0.0, noise, size=(len(pts), 3))
    xyz = xyz @ _rot_random(rng).T
    return Chain(_pdb_round_fast(xyz).astype(np.float32),
                 np.frombuffer("".join(seq).encode(), dtype=np.uint8).copy(), name, na=True)


def na_moved_copy(rng: np.random.Generator, tmpl: Chain, sigma: float, name: str) -> Chain:
    """A rigidly moved copy of a nucleic-acid chain with Gaussian noise."""
    xyz = tmpl.xyz.astype(np.float64) @ _rot_random(rng).T + rng.uniform(-20, 20, size=3)
    xyz = xyz + rng.normal(0.0, sigma, size=xyz.shape)
    return Chain(_pdb_round_fast(xyz).astype(np.float32), tmpl.seq.copy(), name, na=True)


def write_pdb(ch: Chain, path: str) -> None:
    """Write a PDB file the reference reader accepts: C-alpha atoms of a
    protein, or C3' atoms of a nucleic acid (residue names "  A" etc., which
    the reader takes for nucleotides).  Residue numbers run 1..9999 and start
    over (the field has four columns), so consecutive residues always differ."""
    lines = []
    for i in range(ch.length):
        x, y, z = (float(v) for v in ch.xyz[i])
        if ch.na:
            lines.append("ATOM  %5d  C3'   %s A%4d    %8.3f%8.3f%8.3f  1.00  0.00           C\n"
                         % (i + 1, chr(int(ch.seq[i])), i % 9999 + 1, x, y, z))
            continue
        res = AA3[chr(int(ch.seq[i]))]
        lines.append("ATOM  %5d  CA  %3s A%4d    %8.3f%8.3f%8.3f  1.00  0.00           C\n"
                     % (i + 1, res, i % 9999 + 1, x, y, z))
    lines.append("TER\nEND\n")
    with open(path, "w") as f:
        f.writelines(lines)


# -------------------------------------------------------------------------
# workload builders (seeded; sizes of the benchmark configurations)

@dataclass
class Workload:
    queries: List[Chain]
    refs: List[Chain]
    seed: int
    desc: str = ""
    homolog_of: List[int] = field(default_factory=list)  # ref -> query or -1


def config0(seed: int = 1, n_refs: int = 1000, qlen: int = 150,
            lmin: int = 50, lmax: int = 500, homolog_frac: float = 0.2) -> Workload:
    """One query of ``qlen`` residues against ``n_refs`` targets U(lmin,lmax);
    ``homolog_frac`` of them homologs (sigma 1-3 A, 0-10% indels)."""
    rng = np.random.default_rng(seed)
    q = random_chains(rng, [qlen], "qry")[0]
    refs: List[Chain] = []
    hom: List[int] = []
    lens = rng.integers(lmin, lmax + 1, size=n_refs)
    rnd = random_chains(rng, lens, "ref")
    for i in range(n_refs):
        if rng.random() < homolog_frac:
            refs.append(homolog(rng, q, float(rng.uniform(1.0, 3.0)),
                                float(rng.uniform(0.0, 0.10)), f"hom{i:06d}"))
            hom.append(0)
        else:
            refs.append(rnd[i])
            hom.append(-1)
    return Workload([q], refs, seed, f"config0 seed={seed}", hom)


def config1(seed: int = 2, n_queries: int = 16, n_refs: int = 200_000,
            family_frac: float = 0.05) -> Workload:
    """16 queries U(80,800) against log-normal targets (median 250,
    sigma_log 0.6, clipped to 30..2000); ``family_frac`` of the targets are
    members of homolog families (10-50 members, sigma 0.5-4 A, <=15% indels)
    seeded from the queries."""
    rng = np.random.default_rng(seed)
    qlens = rng.integers(80, 801, size=n_queries)
    queries = random_chains(rng, qlens, "qry")
    lens = np.clip(np.round(rng.lognormal(math.log(250.0), 0.6, size=n_refs)), 30, 2000).astype(int)
    refs = random_chains(rng, lens, "ref")
    hom = [-1] * n_refs
    n_fam_members = int(family_frac * n_refs)
    pos = rng.permutation(n_refs)
    k = 0
    while k < n_fam_members:
        fsize = int(rng.integers(10, 51))
        qi = int(rng.integers(0, n_queries))
        for _ in range(fsize):
            if k >= n_fam_members:
                break
            ri = int(pos[k])
            refs[ri] = homolog(rng, queries[qi], float(rng.uniform(0.5, 4.0)),
                               float(rng.uniform(0.0, 0.15)), f"fam{ri:06d}")
            hom[ri] = qi
            k += 1
    return Workload(queries, refs, seed, f"config1 seed={seed}", hom)


def config4(seed: int = 4, n: int = 20_000, family_frac: float = 0.3,
            family_size: int = 10) -> Workload:
    """The all-against-all clustering set: ``n`` structures, log-normal
    lengths (median 220, sigma_log 0.6) clipped to 40..1,200; ``family_frac``
    of them in families of ``family_size`` (a random chain and noisy copies,
    sigma 0.5-3 A, <=10% indels), placed at random positions; names
    s0000000.. in list order.  The structures are returned as ``queries``
    (a clustering run aligns the set against itself)."""
    rng = np.random.default_rng(seed)
    lens = np.clip(np.round(rng.lognormal(math.log(220.0), 0.6, size=n)), 40, 1200).astype(int)
    chains = random_chains(rng, lens, "s")
    nfam = int(family_frac * n) // family_size
    pos = rng.permutation(n)
    hom = [-1] * n
    k = 0
    for f in range(nfam):
        base = chains[int(pos[k])]
        hom[int(pos[k])] = f
        k += 1
        for _ in range(family_size - 1):
            ri = int(pos[k])
            chains[ri] = homolog(rng, base, float(rng.uniform(0.5, 3.0)),
                                 float(rng.uniform(0.0, 0.10)), "s")
            hom[ri] = f
            k += 1
    for i, c in enumerate(chains):
        c.name = "s%07d" % i
    return Workload(chains, [], seed, f"config4 seed={seed} n={n}", hom)


def _rot_small(rng: np.random.Generator, max_deg: float) -> np.ndarray:
    """Rotation by a uniform angle in [0, max_deg] about a random axis."""
    ax = rng.normal(size=3)
    ax /= np.linalg.norm(ax)
    th = math.radians(float(rng.uniform(0.0, max_deg)))
    K = np.array([[0, -ax[2], ax[1]], [ax[2], 0, -ax[0]], [-ax[1], ax[0], 0]])
    return np.eye(3) + math.sin(th) * K + (1 - math.cos(th)) * (K @ K)


def assembly(rng: np.random.Generator, length: int, name: str) -> Tuple[Chain, List[int]]:
    """A multi-domain chain of about ``length`` residues: 100-400-residue
    domains, each placed by a random rigid transform 20-60 A from the
    previous one.  Returns the chain and its domain lengths."""
    dl: List[int] = []
    while sum(dl) < length:
        dl.append(int(min(rng.integers(100, 401), max(length - sum(dl), 1))))
    doms = random_chains(rng, dl, name + "_d")
    parts, centre = [], np.zeros(3)
    for d in doms:
        x = d.xyz.astype(np.float64)
        x = (x - x.mean(axis=0)) @ _rot_random(rng).T
        step = rng.normal(size=3)
        step *= float(rng.uniform(20.0, 60.0)) / np.linalg.norm(step)
        centre = centre + step
        parts.append(x + centre)
    xyz = np.concatenate(parts, axis=0)
    seq = np.concatenate([d.seq for d in doms])
    return Chain(_pdb_round_fast(xyz), seq, name), dl


def assembly_partner(rng: np.random.Generator, ch: Chain, domains: Sequence[int],
                     name: str, max_deg: float = 30.0, sigma: float = 1.5) -> Chain:
    """The long-chain partner: every domain rigidly perturbed (rotation
    about its centre up to ``max_deg``), then Gaussian noise ``sigma``."""
    x = ch.xyz.astype(np.float64).copy()
    o = 0
    for L in domains:
        c = x[o:o + L].mean(axis=0)
        x[o:o + L] = (x[o:o + L] - c) @ _rot_small(rng, max_deg).T + c + rng.normal(0, 1.0, 3)
        o += L
    x += rng.normal(0.0, sigma, size=x.shape)
    x = (x - x.mean(axis=0)) @ _rot_random(rng).T
    return Chain(_pdb_round_fast(x), ch.seq.copy(), name)


def config2(seed: int = 3, lengths: Sequence[int] = (5000, 8000, 12000, 16000, 20000,
                                                     25000, 30000, 37860)) -> Workload:
    """Long-chain pairs: for each length an assembly of 100-400-residue
    domains and its partner (per-domain rotations <= 30 deg, sigma 1.5 A).
    Query i pairs with reference i."""
    rng = np.random.default_rng(seed)
    qs, rs = [], []
    for i, L in enumerate(lengths):
        q, dl = assembly(rng, int(L), f"asm{i:02d}")
        qs.append(q)
        rs.append(assembly_partner(rng, q, dl, f"prt{i:02d}"))
    return Workload(qs, rs, seed, f"config2 seed={seed}", list(range(len(lengths))))


# -------------------------------------------------------------------------
# SoA packing (the layout the C-ABI consumes)

@dataclass
class SoA:
    """Structure-of-arrays block: lengths, prefix offsets, x/y/z, residues."""
    lens: np.ndarray      # (n,) int32
    offs: np.ndarray      # (n,) int32 exclusive prefix sums
    x: np.ndarray         # (N,) float32
    y: np.ndarray
    z: np.ndarray
    rsd: np.ndarray       # (N,) uint8 residue letters
    mol: np.ndarray       # (n,) int32 molecule type (0 protein, 1 nucleic acid)

    @property
    def n(self) -> int:
        return int(self.lens.shape[0])

    @property
    def total(self) -> int:
        return int(self.x.shape[0])


def pack(chains: Sequence[Chain]) -> SoA:
    lens = np.array([c.length for c in chains], dtype=np.int32)
    offs = np.zeros_like(lens)
    if len(lens) > 1:
        offs[1:] = np.cumsum(lens[:-1])
    xyz = np.concatenate([c.xyz for c in chains], axis=0) if chains else np.zeros((0, 3), np.float32)
    rsd = np.concatenate([c.seq for c in chains]) if chains else np.zeros(0, np.uint8)
    return SoA(lens, offs,
               np.ascontiguousarray(xyz[:, 0], dtype=np.float32),
               np.ascontiguousarray(xyz[:, 1], dtype=np.float32),
               np.ascontiguousarray(xyz[:, 2], dtype=np.float32),
               np.ascontiguousarray(rsd, dtype=np.uint8),
               np.array([1 if c.na else 0 for c in chains], dtype=np.int32))


def write_dirs(wl: Workload, qdir: str, rdir: str) -> None:
    os.makedirs(qdir, exist_ok=True)
    os.makedirs(rdir, exist_ok=True)
    for c in wl.queries:
        write_pdb(c, os.path.join(qdir, c.name + ".pdb"))
    for c in wl.refs:
        write_pdb(c, os.path.join(rdir, c.name + ".pdb"))
