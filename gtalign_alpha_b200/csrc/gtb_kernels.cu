// gtb_kernels.cu -- sm_100a kernels of the per-pair superposition search.
//
// Work decomposition (one launch covers every pair of a batch):
//  * seed (stage 1, fragment search): one CTA per pair (a long pair's
//    offsets are split over several CTAs, 512 each), one thread per diagonal
//    offset; each thread runs the whole covariance -> rotation -> score ->
//    threshold loop of its offset sequentially and keeps its best; the CTA
//    reduces (max score, lowest offset index), across CTAs through a packed
//    64-bit atomic maximum.
//  * refinement (every fragment-based superposition refinement): pairs taken
//    from a work list sorted by position count; 16 lanes per pair (32 after
//    the --pre-score filter, 64 warps for pairs of 1,536+ positions) take the
//    pair's admissible (fragment position, fragment length) variants from a
//    pool and advance one pass over the positions at a time; the lanes
//    reduce (max score, lowest variant index).  The distance-threshold
//    covariance pass of iteration k+1 is fused into the scoring pass of
//    iteration k.
//  * DP: pairs from a work list (largest matrices first), one warp per pair;
//    the warp sweeps strips of 32*R rows along anti-diagonals (R rows per
//    lane, register-blocked), left/up/diagonal values move between lanes by
//    shuffles, each lane packs the 2-bit directions of its cells into
//    traceback words.  A long pair's strips run as a wavefront over several
//    single-warp CTAs (cooperative launch, bounded waits on progress counters).
//  * traceback, alignment rows, bookkeeping: one thread per pair.
// All floating-point reductions are sequential per thread in forward position
// order (blocks of BLK positions, Neumaier-compensated), so results do not
// depend on the launch geometry.
#include <algorithm>
#include <type_traits>
#include "gtb200.h"
#include "gtb_device.cuh"
#include "gtb_kernels.cuh"
#include "gtb_gonnet.h"

namespace gtb {

// Residue exchange scores of the --add-search-by-ss DP (log2 Gonnet ratios
// over the letters A..Z, built on the host by gtb_gonnet_scores); a global
// array read through L1: the lanes of a warp look up different residues.
__device__ float g_gonnet[GTB_GONNET_NA * GTB_GONNET_NA];
constexpr float DPSS_C = -1048576.0f;     // offset of a diagonally reached cell
constexpr float DPSS_CMP = -524288.0f;    // stored values below this carry it

__device__ __forceinline__ float gonnet(unsigned char a, unsigned char b) {
    return ('A' <= a && a <= 'Z' && 'A' <= b && b <= 'Z')
               ? __ldg(g_gonnet + (a - 'A') * GTB_GONNET_NA + (b - 'A')) : 0.f;
}


#define GTB_LAUNCHED(T) do { if ((T).launches) (*(T).launches)++; } while (0)

void KTimer::begin(int f, cudaStream_t st) {
    if (used + 2 > ev.size()) {
        for (int k = 0; k < 64; k++) {
            cudaEvent_t e;
            if (cudaEventCreate(&e) != cudaSuccess) return;
            ev.push_back(e);
        }
    }
    if (fam.size() < ev.size() / 2) fam.resize(ev.size() / 2);
    fam[used / 2] = f;
    cudaEventRecord(ev[used], st);
}

void KTimer::end(cudaStream_t st) {
    if (used + 2 > ev.size()) return;       // begin could not create events
    cudaEventRecord(ev[used + 1], st);
    used += 2;
}

cudaError_t KTimer::collect(float* ms) {
    cudaError_t e = cudaSuccess;
    for (size_t k = 0; k + 1 < used; k += 2) {
        float t = 0.f;
        cudaError_t r = cudaEventElapsedTime(&t, ev[k], ev[k + 1]);
        if (r == cudaSuccess) ms[fam[k / 2]] += t;
        else if (e == cudaSuccess) e = r;
    }
    used = 0;
    return e;
}

KTimer::~KTimer() {
    for (cudaEvent_t e : ev) cudaEventDestroy(e);
}

// algorithmic work counters (Bat::work): one atomic per caller, spread over
// WORK_SLOTS addresses by CTA
__device__ __forceinline__ void work_add(const Bat& T, int kind, unsigned long long v) {
    if (T.work && v)
        atomicAdd(T.work + kind * WORK_SLOTS + (blockIdx.x & (WORK_SLOTS - 1)), v);
}

// the transform a DP of pair i uses (DpTfm)
__device__ __forceinline__ const float* dp_tfm(const Bat& T, int i, int tfmsrc) {
    if (tfmsrc == DP_TFM_GRAND) return T.tfm_gr + i * 12;
    if (tfmsrc == DP_TFM_ALT) return T.f3alt + ((long long)i * T.f3br + T.alt_rci) * 12;
    if (tfmsrc == DP_TFM_2ND) return T.tfm_2nd + i * 12;
    return T.tfm_ib + i * 12;
}
// the detailed search's branch T.alt_rci of pair i is empty
__device__ __forceinline__ bool alt_empty(const Bat& T, int i) {
    return T.f3ok && T.alt_rci >= 0 && !T.f3ok[(long long)i * T.f3br + T.alt_rci];
}

__device__ __forceinline__ int pair_qi(const Blk& B, const Bat& T, int i) {
    return (int)((T.p0 + i) / B.nr);
}
__device__ __forceinline__ int pair_ri(const Blk& B, const Bat& T, int i) {
    return (int)((T.p0 + i) % B.nr);
}

// ---------------------------------------------------------------------------
// secondary structure: MpSecStr.cpp:26-118 / MpSecStr.h:218-249
__device__ __forceinline__ float ss_dst(const float* x, const float* y, const float* z, int i, int j) {
    float dx = __fsub_rn(x[i], x[j]), dy = __fsub_rn(y[i], y[j]), dz = __fsub_rn(z[i], z[j]);
    float a = __fmul_rn(dx, dx), b = __fmul_rn(dy, dy), c = __fmul_rn(dz, dz);
    return __fsqrt_rn(__fadd_rn(__fadd_rn(a, b), c));
}

__global__ void k_secstr(char* ss, const float* X, const float* Y, const float* Z,
                         const int* len, const int* off, const int* mol, int nstr) {
    int si = blockIdx.x;
    if (si >= nstr) return;
    int L = len[si];
    const float* x = X + off[si];
    const float* y = Y + off[si];
    const float* z = Z + off[si];
    char* s = ss + off[si];
    int prot = mol ? (mol[si] == 0) : 1;
    for (int p = threadIdx.x; p < L; p += blockDim.x) {
        char c = ' ';
        if (prot && p >= 2 && p + 2 < L) {
            float d13 = ss_dst(x, y, z, p - 2, p);
            float d14 = ss_dst(x, y, z, p - 2, p + 1);
            float d15 = ss_dst(x, y, z, p - 2, p + 2);
            float d24 = ss_dst(x, y, z, p - 1, p + 1);
            float d25 = ss_dst(x, y, z, p - 1, p + 2);
            float d35 = ss_dst(x, y, z, p, p + 2);
            float e = 2.1f;
            if (fabsf(d15 - 6.37f) < e && fabsf(d14 - 5.18f) < e && fabsf(d25 - 5.18f) < e &&
                fabsf(d13 - 5.45f) < e && fabsf(d24 - 5.45f) < e && fabsf(d35 - 5.45f) < e)
                c = 'h';
            else {
                e = 1.42f;
                if (fabsf(d15 - 13.0f) < e && fabsf(d14 - 10.4f) < e && fabsf(d25 - 10.4f) < e &&
                    fabsf(d13 - 6.1f) < e && fabsf(d24 - 6.1f) < e && fabsf(d35 - 6.1f) < e)
                    c = 'e';
                else if (d15 < 8.0f)
                    c = 't';
            }
        }
        s[p] = c;
    }
}

void launch_secstr(char* ss, const float* x, const float* y, const float* z,
                   const int* len, const int* off, const int* mol, int nstr,
                   cudaStream_t st, long long* launches) {
    if (nstr <= 0) return;
    k_secstr<<<nstr, 128, 0, st>>>(ss, x, y, z, len, off, mol, nstr);
    if (launches) (*launches)++;
}

// ---------------------------------------------------------------------------
__global__ void k_pack4(float4* out, const float* x, const float* y, const float* z, long long n) {
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = make_float4(x[i], y[i], z[i], 0.f);
}

void launch_pack4(float4* out, const float* x, const float* y, const float* z, long long n,
                  cudaStream_t st) {
    if (n <= 0) return;
    k_pack4<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(out, x, y, z, n);
}

__global__ void k_pack4s(float4* out, const float* x, const float* y, const float* z,
                         const int* off, const int* len, const int* coff, int n) {
    int si = blockIdx.x;
    if (si >= n) return;
    int o = off[si], L = len[si], c = coff[si];
    for (int p = threadIdx.x; p < L; p += blockDim.x)
        out[c + p] = make_float4(x[o + p], y[o + p], z[o + p], 0.f);
}

void launch_pack4_structs(float4* out, const float* x, const float* y, const float* z,
                          const int* off, const int* len, const int* coff, int n,
                          cudaStream_t st) {
    if (n <= 0) return;
    k_pack4s<<<n, 128, 0, st>>>(out, x, y, z, off, len, coff, n);
}

// ---------------------------------------------------------------------------
// pair initialisation: MpStage1.cpp:28-167
// the clustering run's prefilter of a pair (CheckMaxCoverage)
__device__ __forceinline__ bool cls_pass(const Blk& B, int qi, int ri) {
    const float lq = (float)B.qlen[qi], lr = (float)B.rlen[ri];
    return B.rtype[ri] < B.clsqend && __fmul_rn(fmaxf(lq, lr), B.clscov) <= fminf(lq, lr);
}

// a thread per node; the residue index is relative to the structure, its SS
// byte at the structure's offset + residue
__global__ void k_pack_nodes(float4* nd, int2* nc, const float* x, const float* y, const float* z,
                             const int* l, const int* r, const int* o, const int* off,
                             const int* len, const char* ss, int nstr) {
    const int s = blockIdx.y;
    if (s >= nstr) return;
    const int L = len[s], a = off[s];
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < L; k += gridDim.x * blockDim.x) {
        const int p = a + k, org = o[p];
        const unsigned w = (unsigned)org | ((unsigned)(unsigned char)ss[a + org] << 16);
        nd[p] = make_float4(x[p], y[p], z[p], __uint_as_float(w));
        nc[p] = make_int2(l[p], r[p]);
    }
}

void launch_pack_nodes(float4* nd, int2* nc, const float* x, const float* y, const float* z,
                       const int* l, const int* r, const int* o, const int* off, const int* len,
                       const char* ss, long long n, int nstr, cudaStream_t st) {
    (void)n;
    for (int s0 = 0; s0 < nstr; s0 += 65535) {
        const int ns = nstr - s0 < 65535 ? nstr - s0 : 65535;
        k_pack_nodes<<<dim3(4, ns), 128, 0, st>>>(nd, nc, x, y, z, l, r, o, off + s0, len + s0, ss, ns);
    }
}

__global__ void k_init(Blk B, Bat T) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= T.np) return;
    int qi = pair_qi(B, T, i), ri = pair_ri(B, T, i);
    // with the --pre-similarity screen or in a clustering run every pair starts
    // filtered, with no molecule-type check (custage1.cu:74-82); a clustering
    // run releases the pairs of its triangle whose lengths can reach the
    // coverage (CheckMaxCoverage, coverage.cu:28-52), and k_presim then
    // releases, of the rest, the ones that pass its screen
    if (B.cls) T.flags[i] = cls_pass(B, qi, ri) ? 0 : CONV_LOWTMSC;
    else T.flags[i] = (B.presim > 0.f || B.qmol[qi] != B.rmol[ri]) ? CONV_LOWTMSC : 0;
    T.grand[i] = 0.f; T.best[i] = 0.f; T.best0[i] = 0.f; T.rmsd32[i] = -1.f;
    T.seedq[i] = 0; T.seedr[i] = 0; T.naln[i] = 0;
    T.sfndx[i] = T.sfpos[i] = T.sfndx_cur[i] = T.sfpos_cur[i] = 0;
#pragma unroll
    for (int f = 0; f < 12; f++) {
        float v = (f == 0 || f == 4 || f == 8) ? 1.f : 0.f;
        T.tfm_ib[i * 12 + f] = v;
        T.tfm_gr[i * 12 + f] = v;
    }
#pragma unroll
    for (int f = 0; f < 16; f++) T.out[i * 16 + f] = (f == 8) ? 9999.9f : 0.f;
#pragma unroll
    for (int f = 0; f < 4; f++) T.err[i * 4 + f] = 0.f;
}

void launch_init(const Blk& B, const Bat& T, cudaStream_t st) {
    k_init<<<(T.np + 127) / 128, 128, 0, st>>>(B, T);
    GTB_LAUNCHED(T);
}

// --pre-similarity (MpStage1.cpp:175-248, PMBatchStrData.inl:37-95; the
// reference's GPU form similarity.cu): a pair passes when some diagonal,
// every 2nd one at least PRESIM_EDGE residues from either end, has an
// ungapped run whose Gonnet scores sum to the threshold or more.  Diagonals
// are numbered over the block's longest query and reference: diagonal di
// starts at query position 2*di or, past the query's last admissible start,
// at reference position ((2*di - (lq - 20)) rounded down to even) + 2.  A
// warp per pair, its lanes on 32 diagonals at a time, each summing its run
// in position order (prefix sum minus the smallest prefix so far).
__global__ void __launch_bounds__(128) k_presim(Blk B, Bat T) {
    const unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const int i = blockIdx.x * 4 + (threadIdx.x >> 5);
    if (i >= T.np) return;                        // the same for the whole warp
    int qi = pair_qi(B, T, i), ri = pair_ri(B, T, i);
    if (B.cls && cls_pass(B, qi, ri)) return;     // released already (similarity.cu:60-65)
    const int ql = B.qlen[qi], rl = B.rlen[ri];
    const unsigned char* qa = B.qa + B.qoff[qi];
    const unsigned char* ra = B.ra + B.roff[ri];
    const int ndiag = (B.qmax + B.rmax - 2 * PRESIM_EDGE) >> 1;
    bool pass = false;
    for (int d0 = 0; d0 < ndiag; d0 += 32) {
        const int di = d0 + lane;
        if (di < ndiag && !pass) {
            int qp = di * 2, rp = 0;
            if (ql - PRESIM_EDGE <= qp) { rp = ((qp - (ql - PRESIM_EDGE)) & ~1) + 2; qp = 0; }
            if (!(ql - PRESIM_EDGE <= qp || rl - PRESIM_EDGE <= rp)) {
                const int n1 = ql - qp < rl ? ql - qp : rl, n2 = rl - rp < ql ? rl - rp : ql;
                const int n = n1 < n2 ? n1 : n2;
                float s = 0.f, mn = 0.f, best = 0.f;
                for (int k = 0; k < n; k++) {
                    s = __fadd_rn(s, gonnet(qa[qp + k], ra[rp + k]));
                    mn = s < mn ? s : mn;
                    const float loc = __fsub_rn(s, mn);
                    best = loc > best ? loc : best;
                }
                pass = B.presim <= best;
            }
        }
        if (__any_sync(FULL, pass)) {
            if (lane == 0) T.flags[i] = 0;
            return;
        }
    }
}

void launch_presim(const Blk& B, const Bat& T, cudaStream_t st) {
    k_presim<<<(T.np + 3) / 4, 128, 0, st>>>(B, T);
    GTB_LAUNCHED(T);
}

// ---------------------------------------------------------------------------
// position spaces: a gapless diagonal from (q0, r0), or DP-aligned pairs
// stored in traceback (reverse) order.
// (The aligned space is read from the coordinates the traceback stored
// with each aligned pair, 6 floats per pair in traceback order.)
struct PairGeom {
    const float4 *q4, *r4;  // the pair's structures, (x, y, z, 0) per residue
    const float2* alc;      // aligned coordinates, reverse order; null: diagonal
    int q0, r0, n;
    __device__ __forceinline__ void at(int k, float& a, float& b, float& c,
                                       float& d, float& e, float& f) const {
        if (alc) {
            const float2* p = alc + 3 * (n - 1 - k);
            float2 u = __ldg(p), v = __ldg(p + 1), w = __ldg(p + 2);
            a = u.x; b = u.y; c = v.x; d = v.y; e = w.x; f = w.y;
        } else {
            float4 u = __ldg(q4 + q0 + k), v = __ldg(r4 + r0 + k);
            a = u.x; b = u.y; c = u.z; d = v.x; e = v.y; f = v.z;
        }
    }
    // bring line `ln` (0..7) of the positions [k, k+32) into L1 ahead of use
    __device__ __forceinline__ void prefetch(int k, int ln) const {
        const char* p;
        if (alc) {
            int hi = n - 1 - k;                       // positions run backwards in memory
            if (hi < 0) return;
            int lo = hi - 31 < 0 ? 0 : hi - 31;
            const char* base = (const char*)(alc + 3 * lo);
            const char* end = (const char*)(alc + 3 * (hi + 1));
            p = base + 128 * ln;
            if (p >= end) return;
        } else {
            if (k >= n) return;
            int k1 = k + 32 < n ? k + 32 : n;         // stay inside the pair's residues
            const char* base = ln < 4 ? (const char*)(q4 + q0 + k) : (const char*)(r4 + r0 + k);
            const char* end = ln < 4 ? (const char*)(q4 + q0 + k1) : (const char*)(r4 + r0 + k1);
            p = base + 128 * (ln & 3);
            if (p >= end) return;
        }
        asm volatile("prefetch.global.L1 [%0];" :: "l"(p));
    }
};

// Every pass below walks its range in blocks of BLK positions (folded into
// the compensated totals after each block); the block boundaries count from
// the start of the range, as in the oracle.
__device__ void cov_range(const PairGeom& G, int k0, int k1, float* v) {
    CovAcc a;
    a.init();
    for (int b0 = k0; b0 < k1; b0 += BLK) {
        int b1 = b0 + BLK < k1 ? b0 + BLK : k1;
#pragma unroll 4
        for (int k = b0; k < b1; k++) {
            float qx, qy, qz, rx, ry, rz;
            G.at(k, qx, qy, qz, rx, ry, rz);
            a.add(qx, qy, qz, rx, ry, rz);
        }
        a.fold();
    }
    a.final(v);
}

__device__ void cov_ext(const PairGeom& G, const float* tfm, float thr, float* v) {
    CovAcc a;
    a.init();
    for (int b0 = 0; b0 < G.n; b0 += BLK) {
        int b1 = b0 + BLK < G.n ? b0 + BLK : G.n;
#pragma unroll 4
        for (int k = b0; k < b1; k++) {
            float qx, qy, qz, rx, ry, rz;
            G.at(k, qx, qy, qz, rx, ry, rz);
            float d = dist2_tf(tfm, qx, qy, qz, rx, ry, rz);
            if (d <= thr) a.add(qx, qy, qz, rx, ry, rz);
        }
        a.fold();
    }
    a.final(v);
}

// three smallest distances; m3mode 0 none, 1 distinct values, 2 multiset
__device__ __forceinline__ void track3(int m3mode, float d, float& m1, float& m2, float& m3) {
    if (m3mode == 2) {
        if (d < m1) { m3 = m2; m2 = m1; m1 = d; }
        else if (d < m2) { m3 = m2; m2 = d; }
        else if (d < m3) m3 = d;
    } else if (m3mode == 1) {
        if (d < m1) { m3 = m2; m2 = m1; m1 = d; }
        else if (d > m1 && d < m2) { m3 = m2; m2 = d; }
        else if (d > m2 && d < m3) m3 = d;
    }
}

// score pass under tfm (chk: only distances within d82 count)
__device__ float score_pass(const PairGeom& G, const float* tfm, float d02, int chk, float d82,
                            int m3mode, float& m3out) {
    float ss = 0.f, sc = 0.f, sb = 0.f;
    float m1 = LARGEDST, m2 = LARGEDST, m3 = LARGEDST;
    for (int b0 = 0; b0 < G.n; b0 += BLK) {
        int b1 = b0 + BLK < G.n ? b0 + BLK : G.n;
#pragma unroll 4
        for (int k = b0; k < b1; k++) {
            float qx, qy, qz, rx, ry, rz;
            G.at(k, qx, qy, qz, rx, ry, rz);
            float d = dist2_tf(tfm, qx, qy, qz, rx, ry, rz);
            if (!chk || d <= d82) sb = __fadd_rn(sb, tmterm(d02, d));
            track3(m3mode, d, m1, m2, m3);
        }
        nfold(ss, sc, sb);
    }
    nfold(ss, sc, sb);
    m3out = m3;
    return __fadd_rn(ss, sc);
}

// fused: score under tfm (chk, m3 tracking) and the covariance of the
// positions with d <= thr (the next pass's threshold when it is known, or
// its most likely value when it is not)
__device__ float score_and_ext(const PairGeom& G, const float* tfm, float d02, int chk, float d82,
                               float thr, float* v, int m3mode, float& m3out) {
    float ss = 0.f, sc = 0.f, sb = 0.f;
    float m1 = LARGEDST, m2 = LARGEDST, m3 = LARGEDST;
    CovAcc a;
    a.init();
    for (int b0 = 0; b0 < G.n; b0 += BLK) {
        int b1 = b0 + BLK < G.n ? b0 + BLK : G.n;
#pragma unroll 2
        for (int k = b0; k < b1; k++) {
            float qx, qy, qz, rx, ry, rz;
            G.at(k, qx, qy, qz, rx, ry, rz);
            float d = dist2_tf(tfm, qx, qy, qz, rx, ry, rz);
            if (!chk || d <= d82) sb = __fadd_rn(sb, tmterm(d02, d));
            track3(m3mode, d, m1, m2, m3);
            if (d <= thr) a.add(qx, qy, qz, rx, ry, rz);
        }
        nfold(ss, sc, sb);
        a.fold();
    }
    nfold(ss, sc, sb);
    a.final(v);
    m3out = m3;
    return __fadd_rn(ss, sc);
}

// every one of the 16 sums changed by less than RM_CONVEPS relative (b strided)
__device__ __forceinline__ int converged16(const float* a, const float* b, int bstr) {
    int cnt = 0;
#pragma unroll
    for (int f = 0; f < 16; f++) {
        float x = a[f], y = b[f * bstr];
        float m = fabsf(x) < fabsf(y) ? fabsf(x) : fabsf(y);
        if (fabsf(__fsub_rn(x, y)) < __fmul_rn(m, RM_CONVEPS)) cnt++;
    }
    return cnt >= 16;
}

// ---------------------------------------------------------------------------
// stage 1 seed: MpStage1.cpp:289-440

// The seed's fused pass: score (no d8 check), the three smallest distinct
// distances, the covariance of d <= thr, and the SEED_K smallest distances
// with their positions (ascending; ties keep the earlier position first).
// When the next threshold turns out to be above thr, the positions within
// it are usually these few (three in almost every case), and their
// covariance is rebuilt from the list instead of another pass.
constexpr int SEED_K = 6;

__device__ float seed_score_ext(const PairGeom& G, const float* tfm, float d02, float thr,
                                float* v, float& m3out, float* kd, int* kk) {
    float ss = 0.f, sc = 0.f, sb = 0.f;
    float m1 = LARGEDST, m2 = LARGEDST, m3 = LARGEDST;
#pragma unroll
    for (int j = 0; j < SEED_K; j++) { kd[j] = LARGEDST; kk[j] = 0; }
    CovAcc a;
    a.init();
    for (int b0 = 0; b0 < G.n; b0 += BLK) {
        int b1 = b0 + BLK < G.n ? b0 + BLK : G.n;
#pragma unroll 2
        for (int k = b0; k < b1; k++) {
            float qx, qy, qz, rx, ry, rz;
            G.at(k, qx, qy, qz, rx, ry, rz);
            float d = dist2_tf(tfm, qx, qy, qz, rx, ry, rz);
            sb = __fadd_rn(sb, tmterm(d02, d));
            {   // three smallest distinct distances, branch-free
                bool c1 = d < m1, c2 = d > m1 && d < m2, c3 = d > m2 && d < m3;
                m3 = (c1 || c2) ? m2 : (c3 ? d : m3);
                m2 = c1 ? m1 : (c2 ? d : m2);
                m1 = c1 ? d : m1;
            }
            if (d < kd[SEED_K - 1]) {
                // insert (d, k) keeping kd ascending
                float cd = d;
                int ck = k;
#pragma unroll
                for (int j = 0; j < SEED_K; j++) {
                    bool sw = cd < kd[j];
                    float td = kd[j];
                    int tk = kk[j];
                    kd[j] = sw ? cd : td; kk[j] = sw ? ck : tk;
                    cd = sw ? td : cd; ck = sw ? tk : ck;
                }
            }
            if (d <= thr) a.add(qx, qy, qz, rx, ry, rz);
        }
        nfold(ss, sc, sb);
        a.fold();
    }
    nfold(ss, sc, sb);
    a.final(v);
    m3out = m3;
    return __fadd_rn(ss, sc);
}

// covariance of the listed positions with kd <= thr, in position order
// with the block folds of a full pass (folding an empty block changes
// nothing); valid when every position with d <= thr is listed.
__device__ void seed_cov_list(const PairGeom& G, const float* kd, const int* kk, float thr,
                              float* v) {
    int sel[SEED_K], m = 0;
#pragma unroll
    for (int j = 0; j < SEED_K; j++)
        if (kd[j] <= thr) sel[m++] = kk[j];
    for (int x = 1; x < m; x++) {            // position order
        int y = sel[x], z = x - 1;
        while (z >= 0 && sel[z] > y) { sel[z + 1] = sel[z]; z--; }
        sel[z + 1] = y;
    }
    CovAcc a;
    a.init();
    int blk = -1;
    for (int x = 0; x < m; x++) {
        int k = sel[x];
        if (blk >= 0 && k / BLK != blk) a.fold();
        blk = k / BLK;
        float qx, qy, qz, rx, ry, rz;
        G.at(k, qx, qy, qz, rx, ry, rz);
        a.add(qx, qy, qz, rx, ry, rz);
    }
    a.final(v);
}

// vis: position visits of the passes made (the algorithmic work count)
__device__ float findfrag_variant(const PairGeom& G, float d02, float d0s, int swap,
                                  unsigned long long& vis) {
    float v[16], tfm[12], m3, best = 0.f;
    float d02s0 = __fmul_rn(d0s, d0s);
    cov_range(G, 0, G.n, v);
    vis += G.n;
    for (int it = 0; it < 3; it++) {
        solve_sums(v, swap, tfm);
        vis += G.n;
        if (it == 2) {
            float sc = score_pass(G, tfm, d02, 0, 0.f, 0, m3);
            if (best < sc) best = sc;
            break;
        }
        float d02s = __fadd_rn(d02s0, (it == 1 ? 1.0f : 0.0f));
        // the next threshold is d02s unless the third-smallest distance is
        // above it: accumulate for d02s while scoring, redo in the rare case
        float kd[SEED_K];
        int kk[SEED_K];
        float sc = seed_score_ext(G, tfm, d02, d02s, v, m3, kd, kk);
        if (best < sc) best = sc;
        float dst32;
        if (LARGEDST_CMP < m3 || m3 < d02s || G.n <= 3) dst32 = d02s;
        else dst32 = __fadd_rn(d02s, __fmul_rn(ceilf(__fmul_rn(__fsub_rn(m3, d02s), 2.0f)), 0.5f));
        if (dst32 != d02s) {
            if (dst32 < kd[SEED_K - 1]) seed_cov_list(G, kd, kk, dst32, v);
            else { cov_ext(G, tfm, dst32, v); vis += G.n; }
        }
        if (v[15] < 1.0f) break;
        if ((int)v[15] == G.n) break;
    }
    return best;
}

__global__ void __launch_bounds__(128) k_findfrag(Blk B, Bat T) {
    const int item = blockIdx.x;
    int i = item, c = 0, nch = 1;
    if (T.ff_pair) {
        if (item >= T.nff) return;
        i = T.ff_pair[item];
        c = T.ff_chunk[item];
        nch = T.ff_nch[i];
    }
    if (i >= T.np) return;
    int flags = T.flags[i];
    if (flags & CONV_LOWTMSC) return;
    int qi = pair_qi(B, T, i), ri = pair_ri(B, T, i);
    int lq = B.qlen[qi], lr = B.rlen[ri];
    const int step = B.stepinit;
    int n1, silo, sihi, prv;
    seed_range(lq, lr, B.qmax, B.qmin, B.rmax, B.rmin, step, n1, silo, sihi, prv);
    const int ml = lq < lr ? lq : lr;
    // this CTA's share of the offsets
    int s0 = silo, s1 = sihi;
    if (nch > 1) {
        const int chunk = T.ff_span > 0 ? T.ff_span : FF_CHUNK;
        s0 = silo + c * chunk;
        s1 = s0 + chunk - 1 < sihi ? s0 + chunk - 1 : sihi;
    }
    float d0 = B.t_d0[ml];
    float d02 = __fmul_rn(d0, d0);
    float d0s = d0s_of(d0);
    int swap = B.symmetric && (lq < lr);
    PairGeom G;
    G.q4 = B.q4 + B.q4off[qi]; G.r4 = B.r4 + B.r4off[ri];
    G.alc = nullptr;
    float lbest = 0.f;
    int lsi = 0x7fffffff;
    unsigned long long vis = 0;
    // offsets handed out one at a time (a thread's offsets still come in
    // increasing order, so its strict-improvement rule keeps the lowest index)
    __shared__ int s_next;
    if (threadIdx.x == 0) s_next = s0 + (int)blockDim.x;
    __syncthreads();
    for (int si = s0 + (int)threadIdx.x; si <= s1; si = atomicAdd(&s_next, 1)) {
        int ab = n1 + si * step;
        int qpos = ab > 0 ? ab : 0;
        int rpos = -ab > 0 ? -ab : 0;
        if (lq <= qpos || lr <= rpos) continue;
        if (lq - qpos < prv || lr - rpos < prv) continue;
        G.q0 = qpos; G.r0 = rpos;
        G.n = (lq - qpos) < (lr - rpos) ? (lq - qpos) : (lr - rpos);
        float b = findfrag_variant(G, d02, d0s, swap, vis);
        if (b > 0.f && lbest < b) { lbest = b; lsi = si; }
    }
    __shared__ float sb[128];
    __shared__ int ssi[128];
    __shared__ unsigned long long s_vis;
    if (threadIdx.x == 0) s_vis = 0;
    sb[threadIdx.x] = lbest;
    ssi[threadIdx.x] = lsi;
    __syncthreads();
    if (T.work) atomicAdd(&s_vis, vis);
    for (int s = blockDim.x >> 1; s > 0; s >>= 1) {
        if ((int)threadIdx.x < s) {
            float o = sb[threadIdx.x + s];
            int os = ssi[threadIdx.x + s];
            if (o > sb[threadIdx.x] || (o == sb[threadIdx.x] && os < ssi[threadIdx.x])) {
                sb[threadIdx.x] = o;
                ssi[threadIdx.x] = os;
            }
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        work_add(T, WK_SEED, s_vis);
        float b = sb[0];
        if (nch > 1) {
            // larger score, then lower offset index, over the pair's CTAs
            if (b > 0.f) {
                unsigned long long key = ((unsigned long long)__float_as_uint(b) << 32) |
                                         (unsigned long long)(0xffffffffu - (unsigned)ssi[0]);
                atomicMax(T.ff_key + i, key);
            }
            return;
        }
        T.best[i] = b;
        if (b > 0.f) {
            int ab = n1 + ssi[0] * step;
            T.seedq[i] = ab > 0 ? ab : 0;
            T.seedr[i] = -ab > 0 ? -ab : 0;
        } else {
            T.seedq[i] = 0;
            T.seedr[i] = 0;
        }
    }
}

// seeds of the pairs split over several CTAs
__global__ void k_findfrag_fin(Blk B, Bat T) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= T.np || T.ff_nch[i] <= 1) return;
    if (T.flags[i] & CONV_LOWTMSC) return;
    unsigned long long key = T.ff_key[i];
    float b = __uint_as_float((unsigned)(key >> 32));
    T.best[i] = b;
    if (b > 0.f) {
        int qi = pair_qi(B, T, i), ri = pair_ri(B, T, i);
        int n1, silo, sihi, prv;
        seed_range(B.qlen[qi], B.rlen[ri], B.qmax, B.qmin, B.rmax, B.rmin, B.stepinit, n1, silo,
                   sihi, prv);
        int si = (int)(0xffffffffu - (unsigned)(key & 0xffffffffu));
        int ab = n1 + si * B.stepinit;
        T.seedq[i] = ab > 0 ? ab : 0;
        T.seedr[i] = -ab > 0 ? -ab : 0;
    } else {
        T.seedq[i] = 0;
        T.seedr[i] = 0;
    }
}

void launch_findfrag(const Blk& B, const Bat& T, cudaStream_t st) {
    KtScope kts(T, KF_SEED, st);
    if (T.ff_pair) {
        cudaMemsetAsync(T.ff_key, 0, (size_t)T.np * sizeof(unsigned long long), st);
        k_findfrag<<<T.nff, 128, 0, st>>>(B, T);
        k_findfrag_fin<<<(T.np + 255) / 256, 256, 0, st>>>(B, T);
        if (T.launches) (*T.launches) += 2;
        return;
    }
    k_findfrag<<<T.np, 128, 0, st>>>(B, T);
    GTB_LAUNCHED(T);
}

// ---------------------------------------------------------------------------
// Refinement work list.  Before each refinement launch the pairs that take
// part (mode's convergence flags clear, a non-empty position space) are
// listed in decreasing order of their position count (buckets of 16), so
// that the pairs sharing a warp have passes of about the same length and
// finished pairs cost nothing.  Pairs left out get the mode's outputs for
// "no variant scored" here.
constexpr int RL_SHIFT = 4;
constexpr int RL_NB = 65536 >> RL_SHIFT;   // buckets; rhist[RL_NB] = list length

// position count of pair i in mode `mode`, or -1 when the pair is skipped
__device__ __forceinline__ int refine_span(const Blk& B, const Bat& T, int mode, int i) {
    int flags = T.flags[i];
    if (mode == RM_DP ? flags != 0 : (flags & CONV_LOWTMSC) != 0) return -1;
    if (mode != RM_INIT) return T.naln[i];
    int qi = pair_qi(B, T, i), ri = pair_ri(B, T, i);
    int lq = B.qlen[qi], lr = B.rlen[ri];
    int sq = T.seedq[i], sr = T.seedr[i];
    if (lq <= sq || lr <= sr) return 0;
    return (lq - sq) < (lr - sr) ? (lq - sq) : (lr - sr);
}

__global__ void k_rlist_count(Blk B, Bat T, int mode) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= T.np) return;
    int n = refine_span(B, T, mode, i);
    if (n >= T.rl_min && T.rl_long) {          // many warps for this pair
        int slot = atomicAdd(T.rl_count, 1);
        if (slot < T.rl_nlmax) { T.rl_long[slot] = i; return; }
    } else if (n >= T.rl_min2 && T.rl_long2) {  // the lower tier
        int slot = atomicAdd(T.rl_count2, 1);
        if (slot < T.rl_nlmax2) { T.rl_long2[slot] = i; return; }
    }
    if (n > 0) {
        atomicAdd(&T.rhist[RL_NB - 1 - (n >> RL_SHIFT)], 1);
        return;
    }
    // no variant: MpStage1.cpp:700-716 with nothing scored
    bool skipped = n < 0;
    if (mode == RM_INIT || mode == RM_DP || (!skipped && (mode == RM_FIN1 || mode == RM_FIN2)))
        T.best[i] = 0.f;
    if (!skipped && mode == RM_FIN1) { T.sfndx[i] = T.sfndx_cur[i]; T.sfpos[i] = T.sfpos_cur[i]; }
}

// exclusive scan of the bucket counts (one CTA of 1024 threads)
__global__ void __launch_bounds__(1024) k_rlist_scan(Bat T) {
    __shared__ int part[1024];
    constexpr int PER = RL_NB / 1024;
    int t = threadIdx.x, loc[PER], s = 0;
#pragma unroll
    for (int j = 0; j < PER; j++) { loc[j] = T.rhist[t * PER + j]; s += loc[j]; }
    part[t] = s;
    __syncthreads();
    for (int o = 1; o < 1024; o <<= 1) {
        int v = t >= o ? part[t - o] : 0;
        __syncthreads();
        part[t] += v;
        __syncthreads();
    }
    int run = part[t] - s;
#pragma unroll
    for (int j = 0; j < PER; j++) { T.rhist[t * PER + j] = run; run += loc[j]; }
    if (t == 1023) T.rhist[RL_NB] = part[1023];
}

// DP work list: the pairs a DP launch works on (flags clear, not on the
// wavefront path), largest matrices first; kept in the same buffers as the
// refinement list (a DP launch is over before the next list is built).
__device__ __forceinline__ int dlist_bucket(const Blk& B, const Bat& T, int i, int skipmode) {
    int skipmask = skipmode == 0 ? (CONV_LOWTMSC | CONV_SCOREDP) : CONV_LOWTMSC;
    if (T.flags[i] & skipmask) return -1;
    if (T.dw_mark && T.dw_mark[i]) return -1;
    if (alt_empty(T, i)) return -1;
    int qi = pair_qi(B, T, i), ri = pair_ri(B, T, i);
    long long cells = (long long)B.qlen[qi] * B.rlen[ri];
    long long b = cells >> 8;
    return RL_NB - 1 - (int)(b < RL_NB - 1 ? b : RL_NB - 1);
}

__global__ void k_dlist_count(Blk B, Bat T, int skipmode) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= T.np) return;
    int b = dlist_bucket(B, T, i, skipmode);
    if (b >= 0) atomicAdd(&T.rhist[b], 1);
}

__global__ void k_dlist_fill(Blk B, Bat T, int skipmode) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= T.np) return;
    int b = dlist_bucket(B, T, i, skipmode);
    if (b >= 0) T.rlist[atomicAdd(&T.rhist[b], 1)] = i;
}

// pair list without any flag of skipmask (every size, wavefront pairs too)
__device__ __forceinline__ int plist_bucket(const Blk& B, const Bat& T, int i, int skipmask) {
    if (T.flags[i] & skipmask) return -1;
    int qi = pair_qi(B, T, i), ri = pair_ri(B, T, i);
    long long b = ((long long)B.qlen[qi] * B.rlen[ri]) >> 8;
    return RL_NB - 1 - (int)(b < RL_NB - 1 ? b : RL_NB - 1);
}
__global__ void k_plist_count(Blk B, Bat T, int skipmask) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= T.np) return;
    int b = plist_bucket(B, T, i, skipmask);
    if (b >= 0) atomicAdd(&T.rhist[b], 1);
}
__global__ void k_plist_fill(Blk B, Bat T, int skipmask) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= T.np) return;
    int b = plist_bucket(B, T, i, skipmask);
    if (b >= 0) T.rlist[atomicAdd(&T.rhist[b], 1)] = i;
}

__global__ void k_rlist_fill(Blk B, Bat T, int mode) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= T.np) return;
    int n = refine_span(B, T, mode, i);
    if ((n >= T.rl_min && T.rl_long) || (n >= T.rl_min2 && T.rl_long2))
        return;                                  // listed by k_rlist_count
    if (n > 0) T.rlist[atomicAdd(&T.rhist[RL_NB - 1 - (n >> RL_SHIFT)], 1)] = i;
}

// Variant list of one pair, enumerated compactly (admissible variants only).
// VK_STAGE (6 fragment lengths x step 40): variant si = fct*6 + ndx is
// admissible when frag_length(n, ndx) >= 1 and 40*fct + fraglen < n + 40
// (MpStage1.cpp:635-641).  VK_P2ONE (phase 2, one length: the phase-1
// winner's, 0 promoted to 1): si in [0, nf), pos = pos1 - nf/2 + si, with
// 0 <= pos and pos + fraglen <= n (MpStageFin.cpp:380-396).  VK_P2ALL (phase
// 2, every length: --refinement 2 in production, 3 in both final phases):
// si = fct*6 + ndx, pos = pos1 - nf/2 + fct, the same bounds
// (covariance_production_dp_refn_complete.cu:381-530,
// covariance_fin_dp_refn_complete.cu:464-630).  VK_LOG (one round of the
// log search, covariance_production_dp_refn_complete.cu:836-880): lengths
// 1..5 at pos = pos1 + step, si = ndx, admissible when 0 <= pos and
// pos + fraglen < n + max(step, 0); a fragment reaching past the end is
// shifted back to end at n.
enum VariantKind { VK_STAGE = 0, VK_P2ONE = 1, VK_P2ALL = 2, VK_LOG = 3 };

struct VariantList {
    int total;
    int cnt[FRAG_NSUB], fl[FRAG_NSUB], lo[FRAG_NSUB];
    int base;                 // phase 2: position of si (or fct) = base + si; log: the round's position
};

// the step of log-search round r: +32, -32, +16, -16, ..., +1, -1
__device__ __forceinline__ int plog_step(int r) {
    int st = 32 >> (r >> 1);
    return (r & 1) ? -st : st;
}

__device__ __forceinline__ void variants_init(VariantList& V, int vk, int n, int maxalnmax,
                                              int sfndx0, int sfpos0, int round) {
    V.total = 0;
    V.base = 0;
#pragma unroll
    for (int d = 0; d < FRAG_NSUB; d++) { V.cnt[d] = 0; V.fl[d] = 0; V.lo[d] = 0; }
    if (n <= 0) return;
    if (vk == VK_STAGE) {
        int NF = (int)ceilf((float)(maxalnmax + FRAG_STEP - MINFRAGLEN) / FRAG_STEP);
#pragma unroll
        for (int d = 0; d < FRAG_NSUB; d++) {
            int fl = frag_length(n, d);
            int c = 0;
            if (fl >= 1) {
                c = (n + FRAG_STEP - fl + FRAG_STEP - 1) / FRAG_STEP;
                if (c > NF) c = NF;
                if (c < 0) c = 0;
            }
            V.fl[d] = fl;
            V.cnt[d] = c;
            V.total += c;
        }
        return;
    }
    if (vk == VK_LOG) {
        int step = plog_step(round);
        int pos = sfpos0 + step;
        int ext = step > 0 ? step : 0;
        V.base = pos;
#pragma unroll
        for (int d = 1; d < FRAG_NSUB; d++) {
            int fl = frag_length(n, d);
            int c = (fl >= 1 && pos >= 0 && pos + fl < n + ext) ? 1 : 0;
            V.fl[d] = fl;
            V.cnt[d] = c;
            V.total += c;
        }
        return;
    }
    int nf = 2 * maxalnmax < FIN_MAXNPOS ? 2 * maxalnmax : FIN_MAXNPOS;
    V.base = sfpos0 - (nf >> 1);                // pos = base + fct
    const int lo = -V.base > 0 ? -V.base : 0;   // pos >= 0
#pragma unroll
    for (int d = 0; d < FRAG_NSUB; d++) {
        bool use = vk == VK_P2ALL || d == (sfndx0 == 0 ? 1 : sfndx0);
        int fl = use ? frag_length(n, d) : 0;
        int c = 0;
        if (fl >= 1) {
            int hi = n - fl - V.base;           // pos + fl <= n
            if (hi > nf - 1) hi = nf - 1;
            c = hi >= lo ? hi - lo + 1 : 0;
        }
        V.fl[d] = fl;
        V.lo[d] = lo;
        V.cnt[d] = c;
        V.total += c;
    }
}

// k-th admissible variant (0 <= k < total) -> (si, length index, position,
// length, first position of the refined fragment); variants are grouped by
// length index, so ties are broken by si, not by k
__device__ __forceinline__ void variants_get(const VariantList& V, int vk, int n, int k,
                                             int& si, int& ndx, int& pos, int& fl, int& kf) {
    // the group is selected inside the unrolled loop (no run-time array index)
    int d = 0, c = V.cnt[0], fcl = V.fl[0], lol = V.lo[0];
#pragma unroll
    for (int e = 1; e < FRAG_NSUB; e++) {
        if (k >= c) { k -= c; d = e; c = V.cnt[e]; fcl = V.fl[e]; lol = V.lo[e]; }
    }
    ndx = d;
    fl = fcl;
    if (vk == VK_STAGE) {
        si = k * FRAG_NSUB + d;
        pos = k * FRAG_STEP;
    } else if (vk == VK_LOG) {
        si = d;
        pos = V.base;
    } else {
        int fct = lol + k;
        si = vk == VK_P2ALL ? fct * FRAG_NSUB + d : fct;
        pos = V.base + fct;
    }
    int delta = pos + fl - n;
    kf = pos - (delta > 0 ? delta : 0);
}

// ---------------------------------------------------------------------------
// Refinement.  RF_LPP lanes share one pair and take the pair's admissible
// variants from a pool in list order; a lane whose variant is done takes
// the next one, so the lanes stay busy while variants last.  All lanes
// advance together one pass at a time (a pass = one sweep of the pair's
// positions); what a lane does in a pass depends on where its variant is
// in the refinement loop of MpStage1.cpp:640-700 (and its copies in
// RefineFragDPKernel and MpStageFin.cpp):
enum PassKind {
    PK_IDLE = 0,    // no variant left for this lane
    PK_FRAG = 1,    // covariance of the fragment [k0, k1)
    PK_SCORE = 2,   // score under tfm, fused with the covariance of d <= thr
    PK_EXT = 3,     // covariance of d <= thr only (iteration 1's threshold
                    // when it differs from the one fused into iteration 0)
    PK_GSCORE = 4,  // score of the variant's best transform with another d0
};

// One pass of one lane.  Blocks of BLK positions are the absolute blocks
// of the position space for every kind, so lanes fold together.
// M3 / FR / SC: whether any lane of the warp tracks the three smallest
// distances, covers a fragment, or scores in this pass; the code for what
// no lane does is left out.
template <bool M3, bool FR, bool SC>
__device__ __forceinline__ float lane_pass_t(const PairGeom& G, int kind, int k0, int k1,
                                             const float* tfm, float d02, int chk, float d82,
                                             float thr, int m3on, float* v, float& m3out, int pl) {
    float ss = 0.f, sc = 0.f, sb = 0.f;
    float m1 = LARGEDST, m2 = LARGEDST, m3 = LARGEDST;
    const bool frag = FR && kind == PK_FRAG;
    const bool scr = SC && (kind == PK_SCORE || kind == PK_GSCORE);
    const bool cov = kind == PK_SCORE || kind == PK_EXT;
    const int n = kind == PK_IDLE ? 0 : (frag ? k1 : G.n);
    CovAcc a;
    a.init();
    for (int b0 = frag ? (k0 & ~(BLK - 1)) : 0; b0 < n; b0 += BLK) {
        int b1 = b0 + BLK < n ? b0 + BLK : n;
        if (pl < 8) G.prefetch(b0 + BLK, pl);    // the next block, one line per lane
#pragma unroll 2
        for (int k = b0; k < b1; k++) {
            float qx, qy, qz, rx, ry, rz;
            G.at(k, qx, qy, qz, rx, ry, rz);
            float d = dist2_tf(tfm, qx, qy, qz, rx, ry, rz);
            // branch-free: adding +0 and zero coordinates leaves the sums unchanged
            if (SC) {
                float tm = tmterm(d02, d);
                sb = __fadd_rn(sb, (scr && (!chk || d <= d82)) ? tm : 0.f);
            }
            if (M3) {
                bool c1 = m3on && d < m1, c2 = m3on && d < m2, c3 = m3on && d < m3;
                m3 = c2 ? m2 : (c3 ? d : m3);
                m2 = c1 ? m1 : (c2 ? d : m2);
                m1 = c1 ? d : m1;
            }
            bool inc = FR ? (frag ? (k0 <= k) : (cov && d <= thr)) : (cov && d <= thr);
            a.add(inc ? qx : 0.f, inc ? qy : 0.f, inc ? qz : 0.f,
                  inc ? rx : 0.f, inc ? ry : 0.f, inc ? rz : 0.f);
            a.n += inc ? 0 : -1;
        }
        nfold(ss, sc, sb);
        a.fold();
    }
    nfold(ss, sc, sb);
    a.final(v);
    m3out = m3;
    return __fadd_rn(ss, sc);
}

__device__ __forceinline__ float lane_pass(const PairGeom& G, int kind, int k0, int k1,
                                           const float* tfm, float d02, int chk, float d82,
                                           float thr, int m3on, float* v, float& m3out, int pl) {
    const unsigned FULL = 0xffffffffu;
    const bool sc = __any_sync(FULL, kind == PK_SCORE || kind == PK_GSCORE);
    const bool m3 = __any_sync(FULL, kind == PK_SCORE && m3on);
    const bool fr = __any_sync(FULL, kind == PK_FRAG);
    if (m3)
        return fr ? lane_pass_t<true, true, true>(G, kind, k0, k1, tfm, d02, chk, d82, thr, m3on, v, m3out, pl)
                  : lane_pass_t<true, false, true>(G, kind, k0, k1, tfm, d02, chk, d82, thr, m3on, v, m3out, pl);
    if (sc)
        return fr ? lane_pass_t<false, true, true>(G, kind, k0, k1, tfm, d02, chk, d82, thr, m3on, v, m3out, pl)
                  : lane_pass_t<false, false, true>(G, kind, k0, k1, tfm, d02, chk, d82, thr, m3on, v, m3out, pl);
    return fr ? lane_pass_t<false, true, false>(G, kind, k0, k1, tfm, d02, chk, d82, thr, m3on, v, m3out, pl)
              : lane_pass_t<false, false, false>(G, kind, k0, k1, tfm, d02, chk, d82, thr, m3on, v, m3out, pl);
}

// One pass of a variant that the 32 lanes of a warp share (the long pairs'
// refinement when few pairs are long).  Lane L sums the positions of block
// cb + L (blocks of BLK positions, the absolute blocks of lane_pass_t) in
// position order, exactly as lane_pass_t sums a block; the block partials
// then go through shared memory and lane f folds field f of every block in
// block order (the same Neumaier folds, the same closing fold), so the sums,
// the score and the three smallest distances equal lane_pass_t's bit for
// bit.  Every lane returns the results.  sm: 32 x 17 floats of this warp.
__device__ float wide_pass(const PairGeom& G, int kind, int k0, int k1, const float* tfm,
                           float d02, int chk, float d82, float thr, int m3on, float* v,
                           float& m3out, int lane, float* sm) {
    const unsigned FULL = 0xffffffffu;
    const bool frag = kind == PK_FRAG;
    const bool scr = kind == PK_SCORE || kind == PK_GSCORE;
    const bool cov = kind == PK_SCORE || kind == PK_EXT;
    const bool trk = kind == PK_SCORE && m3on;
    const int n = kind == PK_IDLE ? 0 : (frag ? k1 : G.n);
    const int bfirst = frag ? (k0 & ~(BLK - 1)) / BLK : 0;
    const int nblk = (n + BLK - 1) / BLK;
    float fs = 0.f, fc = 0.f;                  // lane f < 16: field f's compensated total
    float m1 = LARGEDST, m2 = LARGEDST, m3 = LARGEDST;
    int cnt = 0;
    for (int cb = bfirst; cb < nblk; cb += 32) {
        const int b = cb + lane;
        float part[16];
#pragma unroll
        for (int f = 0; f < 16; f++) part[f] = 0.f;
        if (b < nblk) {
            const int p0 = b * BLK, p1 = p0 + BLK < n ? p0 + BLK : n;
            for (int k = p0; k < p1; k++) {
                float qx, qy, qz, rx, ry, rz;
                G.at(k, qx, qy, qz, rx, ry, rz);
                float d = dist2_tf(tfm, qx, qy, qz, rx, ry, rz);
                if (scr) part[15] = __fadd_rn(part[15], (!chk || d <= d82) ? tmterm(d02, d) : 0.f);
                if (trk) {
                    bool c1 = d < m1, c2 = d < m2, c3 = d < m3;
                    m3 = c2 ? m2 : (c3 ? d : m3);
                    m2 = c1 ? m1 : (c2 ? d : m2);
                    m1 = c1 ? d : m1;
                }
                bool inc = frag ? (k0 <= k) : (cov && d <= thr);
                const float ax = inc ? qx : 0.f, ay = inc ? qy : 0.f, az = inc ? qz : 0.f;
                const float bx = inc ? rx : 0.f, by = inc ? ry : 0.f, bz = inc ? rz : 0.f;
                part[0] = __fmaf_rn(ax, bx, part[0]); part[1] = __fmaf_rn(ax, by, part[1]);
                part[2] = __fmaf_rn(ax, bz, part[2]); part[3] = __fmaf_rn(ay, bx, part[3]);
                part[4] = __fmaf_rn(ay, by, part[4]); part[5] = __fmaf_rn(ay, bz, part[5]);
                part[6] = __fmaf_rn(az, bx, part[6]); part[7] = __fmaf_rn(az, by, part[7]);
                part[8] = __fmaf_rn(az, bz, part[8]);
                part[9] = __fadd_rn(part[9], ax); part[10] = __fadd_rn(part[10], ay);
                part[11] = __fadd_rn(part[11], az); part[12] = __fadd_rn(part[12], bx);
                part[13] = __fadd_rn(part[13], by); part[14] = __fadd_rn(part[14], bz);
                cnt += inc ? 1 : 0;
            }
        }
        __syncwarp();
#pragma unroll
        for (int f = 0; f < 16; f++) sm[lane * 17 + f] = part[f];
        __syncwarp();
        if (lane < 16) {
            const int nb = nblk - cb < 32 ? nblk - cb : 32;
            for (int L = 0; L < nb; L++) {
                float bb = sm[L * 17 + lane];
                nfold(fs, fc, bb);
            }
        }
    }
    // the closing fold of lane_pass_t (score) and of CovAcc::final (sums)
    if (lane < 16) {
        float z = 0.f;
        nfold(fs, fc, z);
    }
    const float tot = __fadd_rn(fs, fc);
#pragma unroll
    for (int f = 0; f < 15; f++) v[f] = __shfl_sync(FULL, tot, f);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) cnt += __shfl_xor_sync(FULL, cnt, o);
    v[15] = (float)cnt;
    // the three smallest distances of the pass (a multiset: merging the
    // lanes' three smallest gives the same three as one sweep)
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const float o1 = __shfl_xor_sync(FULL, m1, o), o2 = __shfl_xor_sync(FULL, m2, o),
                    o3 = __shfl_xor_sync(FULL, m3, o);
        const float x[3] = {o1, o2, o3};
#pragma unroll
        for (int e = 0; e < 3; e++) {
            const float d = x[e];
            bool c1 = d < m1, c2 = d < m2, c3 = d < m3;
            m3 = c2 ? m2 : (c3 ? d : m3);
            m2 = c1 ? m1 : (c2 ? d : m2);
            m1 = c1 ? d : m1;
        }
    }
    m3out = m3;
    __syncwarp();
    return __shfl_sync(FULL, tot, 15);
}

// The pair's result of a refinement launch (MpStage1.cpp:700-716 and the
// final/production copies): winner score, transform and fragment, or the
// "nothing scored" outputs.  tb: the winner's transform, stride tstr.
template <int MODE>
__device__ __forceinline__ void refine_commit(const Blk& B, const Bat& T, int i, int lq, int lr,
                                              bool havewin, float wb, float lgbest, int wndx,
                                              int wpos, const float* tb, int tstr) {
    if (MODE == RM_PROD1 || MODE == RM_PROD2 || MODE == RM_PLOG) {
        if (!havewin) return;
        float grand = T.grand[i];
        bool write = (MODE == RM_PROD1) || (grand < wb);
        if (write) {
            T.grand[i] = wb;
            float bs = wb, gb = lgbest;
            if ((float)lr < (float)lq) { float t = bs; bs = gb; gb = t; }
            T.out[i * 16 + 9] = __fdiv_rn(bs, (float)lq);
            T.out[i * 16 + 10] = __fdiv_rn(gb, (float)lr);
            T.out[i * 16 + 11] = B.t_d0fin[lq];
            T.out[i * 16 + 12] = B.t_d0fin[lr];
#pragma unroll
            for (int f = 0; f < 12; f++) T.tfm_gr[i * 12 + f] = tb[f * tstr];
            if (MODE == RM_PROD1) { T.sfndx[i] = wndx; T.sfpos[i] = wpos; }
            if (MODE == RM_PLOG) T.sfpos[i] = wpos;   // the search moves to the round's position
        }
        return;
    }
    T.best[i] = havewin ? wb : 0.f;
    if (havewin) {
#pragma unroll
        for (int f = 0; f < 12; f++) T.tfm_ib[i * 12 + f] = tb[f * tstr];
        if (T.grand[i] < wb) {
            T.grand[i] = wb;
#pragma unroll
            for (int f = 0; f < 12; f++) T.tfm_gr[i * 12 + f] = tb[f * tstr];
        }
    }
    if (MODE == RM_FIN1) {
        // the winner's fragment, or the previous one when no variant scored
        int nd = havewin ? wndx : T.sfndx_cur[i];
        int np_ = havewin ? wpos : T.sfpos_cur[i];
        T.sfndx_cur[i] = nd; T.sfpos_cur[i] = np_;
        T.sfndx[i] = nd; T.sfpos[i] = np_;
    }
}

// RF_LPP lanes per pair: 16 (two pairs per warp) where most pairs of a
// batch take part; 32 where few do (after the --pre-score filter), which
// shortens the launches whose time is that of their slowest pair.
// Warps per CTA: 4 (1 and 2, with an SM refilling a finished warp's slot at
// once, measured the same on the benchmark step: the concurrent sub-batch
// streams fill those slots already).
constexpr int RF_WARPS_SHORT = 4;
constexpr int RF_WARPS_LONG = RLW_CTA_WARPS;

// LONG: the pairs with at least RL_LONG positions, RLW_CTAS CTAs each; every
// warp of them takes the pair's variants from one counter in global memory
// and leaves its best variant as a candidate; k_refine_long_fin picks the
// pair's winner among them.
// One slot of a refinement launch: a short pair (slot of the length-sorted
// list) or, LONG, warp `wlong` of the warps working on long pair `slot`.
// WIDE (long pairs only): a warp works on one variant at a time, its lanes
// sharing the passes (wide_pass); otherwise every lane has a variant.
template <int MODE, int RF_LPP, bool LONG, bool WIDE = false>
__device__ __forceinline__ void refine_slot(const Blk& B, const Bat& T, int slot, int wlong) {
    constexpr int RF_WARPS = LONG ? RF_WARPS_LONG : RF_WARPS_SHORT;
    static_assert(!WIDE || (LONG && RF_LPP == 32), "a wide pass is a long pair's warp");
    __shared__ float s_wide[WIDE ? 17 * RF_WARPS * 32 : 1];   // block partials of wide passes
    __shared__ float s_last[16 * RF_WARPS * 32];   // previous iteration's sums
    __shared__ float s_tb[12 * RF_WARPS * 32];     // best transform of the current variant
    __shared__ float s_tbest[12 * RF_WARPS * 32];  // best transform over the lane's variants
    const unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const int sub = lane / RF_LPP;
    const unsigned smask = RF_LPP == 32 ? 0xffffffffu : ((1u << (RF_LPP & 31)) - 1u) << (sub * RF_LPP);
    const bool valid = LONG ? slot < *T.rl_count : slot < T.rhist[RL_NB];
    if (__ballot_sync(FULL, valid) == 0) return;
    const int i = valid ? (LONG ? T.rl_long[slot] : T.rlist[slot]) : 0;
    const int str = RF_WARPS * 32;
    float* last = s_last + threadIdx.x;
    float* tbs = s_tb + threadIdx.x;
    float* tbest = s_tbest + threadIdx.x;
    int qi = pair_qi(B, T, i), ri = pair_ri(B, T, i);
    int lq = B.qlen[qi], lr = B.rlen[ri];
    int ml = lq < lr ? lq : lr;
    int swap = B.symmetric && (lq < lr);
    PairGeom G;
    G.q4 = B.q4 + B.q4off[qi]; G.r4 = B.r4 + B.r4off[ri];
    if (MODE == RM_INIT) {
        int sq = T.seedq[i], sr = T.seedr[i];
        G.alc = nullptr;
        G.q0 = sq; G.r0 = sr;
        if (lq <= sq || lr <= sr) G.n = 0;
        else G.n = (lq - sq) < (lr - sr) ? (lq - sq) : (lr - sr);
    } else {
        G.alc = (const float2*)(T.alc + 6 * T.off_aln[i]);
        G.q0 = G.r0 = 0;
        G.n = T.naln[i];
    }
    if (!valid) G.n = 0;
    const int n = G.n;
    const bool prod = (MODE == RM_PROD1 || MODE == RM_PROD2 || MODE == RM_PLOG);
    const bool phase2 = (MODE == RM_FIN2 || MODE == RM_PROD2 || MODE == RM_PLOG);
    const int vk = MODE == RM_PLOG ? VK_LOG
                 : MODE == RM_FIN2 ? (B.refinement == GTB_REFINEMENT_FULLA ? VK_P2ALL : VK_P2ONE)
                 : MODE == RM_PROD2 ? (B.refinement >= GTB_REFINEMENT_FULL ? VK_P2ALL : VK_P2ONE)
                 : VK_STAGE;
    const float d0 = prod ? B.t_d0fin[ml] : B.t_d0[ml];
    const float d02 = __fmul_rn(d0, d0);
    const float d82 = B.t_d82[ml];
    const int chk = prod ? 0 : 1;
    // the log search carries the best score so far (phase 1's to begin with)
    // into every variant; the other modes start each variant afresh
    const float best_init = (MODE == RM_INIT || MODE == RM_DP) ? 0.f
                          : MODE == RM_PLOG ? T.grand[i] : -1.f;
    const int maxalnmax = B.qmax < B.rmax ? B.qmax : B.rmax;
    const float d0s = d0s_of(d0);
    const float d0sm = __fsub_rn(d0s, 1.0f);
    const float d02s = __fmul_rn(d0sm, d0sm);       // iteration 1's usual threshold
    const float d0sp = __fadd_rn(d0s, 1.0f);
    const float thr2 = __fmul_rn(d0sp, d0sp);       // threshold of iterations >= 2
    const bool gscore = prod && lq != lr;           // also scored by the longer length
    float g02 = 0.f;
    if (gscore) { float g0 = B.t_d0fin[lq > lr ? lq : lr]; g02 = __fmul_rn(g0, g0); }
    VariantList V;
    variants_init(V, vk, n, maxalnmax, phase2 ? T.sfndx[i] : 0, phase2 ? T.sfpos[i] : 0, T.plog_round);
    if (MODE == RM_PROD1 && (lane % RF_LPP) == 0 && V.total > 0 && wlong == 0) {
        // RMSD over the whole alignment (variant 0: fragment [0, n)) from
        // compensated FP32 sums, MpStageFin.cpp production phase 1
        int s0, nd0, ps0, fl0, kf0;
        variants_get(V, vk, n, 0, s0, nd0, ps0, fl0, kf0);
        CovAcc a;
        a.init();
        float sq[6], cq[6], bq[6];
#pragma unroll
        for (int f = 0; f < 6; f++) { sq[f] = 0.f; cq[f] = 0.f; bq[f] = 0.f; }
        int blk = 0;
        for (int kk = kf0; kk < kf0 + fl0; kk++) {
            float qx, qy, qz, rx, ry, rz;
            G.at(kk, qx, qy, qz, rx, ry, rz);
            a.add(qx, qy, qz, rx, ry, rz);
            bq[0] = __fmaf_rn(qx, qx, bq[0]); bq[1] = __fmaf_rn(qy, qy, bq[1]); bq[2] = __fmaf_rn(qz, qz, bq[2]);
            bq[3] = __fmaf_rn(rx, rx, bq[3]); bq[4] = __fmaf_rn(ry, ry, bq[4]); bq[5] = __fmaf_rn(rz, rz, bq[5]);
            if (++blk == BLK) {
                a.fold();
#pragma unroll
                for (int f = 0; f < 6; f++) nfold(sq[f], cq[f], bq[f]);
                blk = 0;
            }
        }
        float vv[16];
        a.final(vv);
        double dv[21];
#pragma unroll
        for (int f = 0; f < 15; f++) dv[f] = (double)vv[f];
#pragma unroll
        for (int f = 0; f < 6; f++) { nfold(sq[f], cq[f], bq[f]); dv[15 + f] = (double)__fadd_rn(sq[f], cq[f]); }
        T.rmsd32[i] = (float)rmsd_from_sums(dv, (double)fl0);
    }
    float lbest = 0.f, lgbest = 0.f;              // this lane's best variant so far
    int lsi = 0x7fffffff, lndx = 0, lpos = 0;
    int kind = PK_IDLE, si = 0, vndx = 0, vpos = 0, k0 = 0, k1 = 0, cit = 0, m3mode = 0, pchk = chk;
    float best = 0.f, thr = 0.f, pd02 = d02;
    float tfm[12];
#pragma unroll
    for (int f = 0; f < 12; f++) tfm[f] = 0.f;
    bool need = true;
    int nextk = 0;                                // the pair's next variant to hand out
    unsigned long long vis = 0;                   // position visits of this lane's passes
    for (;;) {
        const unsigned nm = __ballot_sync(FULL, need) & smask;
        if (WIDE && nm) {                         // one variant for the whole warp
            int base = 0;
            if (lane == 0) base = atomicAdd(T.rl_next + slot, 1);
            const int kv = __shfl_sync(FULL, base, 0);
            need = false;
            kind = PK_IDLE;
            if (kv < V.total) {
                int fl, kf;
                variants_get(V, vk, n, kv, si, vndx, vpos, fl, kf);
                if (MODE == RM_DP && T.vskip && si < 32 * F3_NSEC &&
                    ((T.vskip[(long long)i * F3_NSEC + (si >> 5)] >> (si & 31)) & 1u)) {
                    need = true;
                } else {
                    kind = PK_FRAG; k0 = kf; k1 = kf + fl;
                    best = best_init; cit = 0;
                }
            }
            if (need) continue;                   // a skipped variant: the next one
        } else if (nm) {
            if (LONG) {                           // the pair's counter, shared by its warps
                int base = 0;
                if (lane == 0) base = atomicAdd(T.rl_next + slot, __popc(nm));
                nextk = __shfl_sync(FULL, base, 0);
            }
            int kv = nextk + __popc(nm & ((1u << lane) - 1u));
            nextk += __popc(nm);
            if (need) {
                need = false;
                kind = PK_IDLE;
                if (kv < V.total) {
                    int fl, kf;
                    variants_get(V, vk, n, kv, si, vndx, vpos, fl, kf);
                    if (MODE == RM_DP && T.vskip && si < 32 * F3_NSEC &&
                        ((T.vskip[(long long)i * F3_NSEC + (si >> 5)] >> (si & 31)) & 1u)) {
                        need = true;       // a variant the detailed search's slots rule out
                    } else {
                        kind = PK_FRAG; k0 = kf; k1 = kf + fl;
                        best = best_init; cit = 0;
                    }
                }
            }
        }
        if (__ballot_sync(FULL, kind != PK_IDLE) == 0) {
            // lanes that passed over a skipped variant take the next one
            if (MODE == RM_DP && T.vskip && __any_sync(FULL, need && nextk < V.total)) continue;
            break;
        }
        float v[16], m3;
        const float sc = WIDE ? wide_pass(G, kind, k0, k1, tfm, pd02, pchk, d82, thr, m3mode, v, m3,
                                          lane, s_wide + (threadIdx.x >> 5) * 32 * 17)
                              : lane_pass(G, kind, k0, k1, tfm, pd02, pchk, d82, thr, m3mode, v, m3,
                                          lane % RF_LPP);
        if (!WIDE || lane == 0)
            vis += kind == PK_IDLE ? 0u : (kind == PK_FRAG ? (unsigned)(k1 - k0) : (unsigned)n);
        bool havev = false, done = false;
        if (kind == PK_FRAG) {
            if (v[15] < 1.0f) done = true;
            else {
#pragma unroll
                for (int f = 0; f < 16; f++) last[f * str] = v[f];
                solve_sums(v, swap, tfm);
                kind = PK_SCORE; thr = d02s; m3mode = 2; cit = 0; pd02 = d02; pchk = chk;
            }
        } else if (kind == PK_SCORE) {
            if (best < sc) {
                best = sc;
#pragma unroll
                for (int f = 0; f < 12; f++) tbs[f * str] = tfm[f];
            }
            havev = true;
            if (cit == 0) {
                // iteration 1's threshold from iteration 0's three smallest distances
                float dst32;
                if (LARGEDST_CMP < m3 || m3 < d02s || n <= 3) dst32 = d02s;
                else {
                    float t = __fadd_rn(d0sm, __fmul_rn(ceilf(__fmul_rn(__fsub_rn(__fsqrt_rn(m3), d0sm), 2.0f)), 0.5f));
                    dst32 = __fmul_rn(t, t);
                }
                if (dst32 != d02s) { kind = PK_EXT; thr = dst32; m3mode = 0; havev = false; }
            }
            cit++;
        } else if (kind == PK_EXT) {
            havev = true;
        } else if (kind == PK_GSCORE) {
            done = true;
        }
        if (havev) {
            if (cit >= NMAXCONVIT + 2 || converged16(v, last, str) || v[15] < 1.0f) done = true;
            else {
#pragma unroll
                for (int f = 0; f < 16; f++) last[f * str] = v[f];
                solve_sums(v, swap, tfm);
                kind = PK_SCORE; thr = thr2; m3mode = 0;
            }
        }
        if (done) {
            if (kind != PK_GSCORE && gscore && best >= 0.f && (MODE != RM_PLOG || best > best_init)) {
                // one more pass: the variant's best transform scored with the
                // d0 of the longer structure
#pragma unroll
                for (int f = 0; f < 12; f++) tfm[f] = tbs[f * str];
                kind = PK_GSCORE; pd02 = g02; pchk = 0; m3mode = 0;
            } else {
                const float gbest = kind == PK_GSCORE ? sc : best;
                if (best > 0.f && (lbest < best || (lbest == best && si < lsi))) {
                    lbest = best; lgbest = gbest; lsi = si; lndx = vndx; lpos = vpos;
#pragma unroll
                    for (int f = 0; f < 12; f++) tbest[f * str] = tbs[f * str];
                }
                need = true;
                kind = PK_IDLE;
            }
        }
    }
    if (T.work) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) vis += __shfl_xor_sync(FULL, vis, o);
        if (lane == 0) work_add(T, WK_REFINE, vis);
    }
    // arg-max over the pair's lanes: larger score, then lower variant index
    float wb = lbest;
    int wsi = lsi;
#pragma unroll
    for (int o = RF_LPP / 2; o > 0; o >>= 1) {
        float ob = __shfl_xor_sync(FULL, wb, o);
        int os = __shfl_xor_sync(FULL, wsi, o);
        if (ob > wb || (ob == wb && os < wsi)) { wb = ob; wsi = os; }
    }
    const bool havewin = wb > 0.f;
    const unsigned wmask = __ballot_sync(FULL, havewin && lsi == wsi) & smask;
    const int wl = wmask ? __ffs(wmask) - 1 : sub * RF_LPP;
    const int wndx = __shfl_sync(FULL, lndx, wl);
    const int wpos = __shfl_sync(FULL, lpos, wl);
    if (!valid) return;
    if (LONG) {
        if (lane == wl) {
            float* c = T.rl_cand + ((long long)slot * (T.rlw_ctas * RF_WARPS_LONG) + wlong) * RLW_CAND;
            c[0] = havewin ? wb : 0.f;
            c[1] = __int_as_float(wsi);
            c[2] = lgbest;
            c[3] = __int_as_float(wndx);
            c[4] = __int_as_float(wpos);
#pragma unroll
            for (int f = 0; f < 12; f++) c[5 + f] = tbest[f * str];
        }
        return;
    }
    if (lane == wl)
        refine_commit<MODE>(B, T, i, lq, lr, havewin, wb, lgbest, wndx, wpos, tbest, str);
}

// LONG: T.rlw_ctas CTAs per long pair; the grid (a multiple of that) walks
// the long pairs listed for this launch.
template <int MODE, int RF_LPP, bool LONG, bool WIDE = false>
__global__ void __launch_bounds__((LONG ? RF_WARPS_LONG : RF_WARPS_SHORT) * 32) k_refine(Blk B, Bat T) {
    if (LONG) {
        const int c = T.rlw_ctas;
        const int wl = (int)(blockIdx.x % c) * RF_WARPS_LONG + (threadIdx.x >> 5);
        const int nlong = *T.rl_count;
        for (int slot = (int)(blockIdx.x / c); slot < nlong; slot += (int)(gridDim.x / c))
            refine_slot<MODE, RF_LPP, LONG, WIDE>(B, T, slot, wl);
    } else {
        constexpr int RF_PPW = 32 / RF_LPP;        // pairs per warp
        const int slot = blockIdx.x * (RF_PPW * RF_WARPS_SHORT) + (threadIdx.x >> 5) * RF_PPW +
                         (int)(threadIdx.x & 31) / RF_LPP;
        refine_slot<MODE, RF_LPP, LONG>(B, T, slot, 0);
    }
}

// the winner of each long pair among its warps' candidates
template <int MODE>
__global__ void k_refine_long_fin(Blk B, Bat T) {
    const unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const int slot = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (slot >= *T.rl_count) return;
    const int i = T.rl_long[slot];
    const float* c0 = T.rl_cand + (long long)slot * (T.rlw_ctas * RF_WARPS_LONG) * RLW_CAND;
    float wb = 0.f;
    int wsi = 0x7fffffff, wk = -1;
    const int nw = T.rlw_ctas * RF_WARPS_LONG;      // the warps that left candidates
    for (int k = lane; k < nw; k += 32) {
        float b = c0[k * RLW_CAND];
        int si = __float_as_int(c0[k * RLW_CAND + 1]);
        if (b > 0.f && (wb < b || (wb == b && si < wsi))) { wb = b; wsi = si; wk = k; }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        float ob = __shfl_xor_sync(FULL, wb, o);
        int os = __shfl_xor_sync(FULL, wsi, o);
        int ok = __shfl_xor_sync(FULL, wk, o);
        if (ob > wb || (ob == wb && os < wsi)) { wb = ob; wsi = os; wk = ok; }
    }
    if (lane != 0) return;
    int qi = pair_qi(B, T, i), ri = pair_ri(B, T, i);
    const bool havewin = wb > 0.f;
    const float* c = c0 + (havewin ? wk : 0) * RLW_CAND;
    refine_commit<MODE>(B, T, i, B.qlen[qi], B.rlen[ri], havewin, wb, c[2], __float_as_int(c[3]),
                        __float_as_int(c[4]), c + 5, 1);
}

template <int LPP, bool LONG, bool WIDE = false>
static void launch_refine_k(int mode, const Blk& B, const Bat& T, cudaStream_t st) {
    constexpr int W = LONG ? RF_WARPS_LONG : RF_WARPS_SHORT;
    // long pairs: at most RLW_GRID CTAs, T.rlw_ctas per pair at a time
    const int nslot = LONG ? std::max(1, std::min(T.rl_nlmax, RLW_GRID / T.rlw_ctas)) : 0;
    const int ng = LONG ? nslot * T.rlw_ctas
                        : (T.np + (32 / LPP) * W - 1) / ((32 / LPP) * W);
    const int nt = W * 32;
    switch (mode) {
        case RM_INIT:  k_refine<RM_INIT, LPP, LONG, WIDE><<<ng, nt, 0, st>>>(B, T); break;
        case RM_DP:    k_refine<RM_DP, LPP, LONG, WIDE><<<ng, nt, 0, st>>>(B, T); break;
        case RM_FIN1:  k_refine<RM_FIN1, LPP, LONG, WIDE><<<ng, nt, 0, st>>>(B, T); break;
        case RM_FIN2:  k_refine<RM_FIN2, LPP, LONG, WIDE><<<ng, nt, 0, st>>>(B, T); break;
        case RM_PROD1: k_refine<RM_PROD1, LPP, LONG, WIDE><<<ng, nt, 0, st>>>(B, T); break;
        case RM_PROD2: k_refine<RM_PROD2, LPP, LONG, WIDE><<<ng, nt, 0, st>>>(B, T); break;
        case RM_PLOG:  k_refine<RM_PLOG, LPP, LONG, WIDE><<<ng, nt, 0, st>>>(B, T); break;
    }
}

// The refinement kernels re-read each pair's positions on every pass: ask
// for the smallest shared-memory carve-out that holds as many CTAs as their
// registers allow (static arrays + the 1 kB each CTA reserves), leaving the
// rest of the SM's 256 kB to L1.
template <int LPP, bool LONG, bool WIDE = false>
static void carve_refine() {
    constexpr int W = LONG ? RF_WARPS_LONG : RF_WARPS_SHORT;
    const void* ks[7] = {(const void*)k_refine<RM_INIT, LPP, LONG, WIDE>, (const void*)k_refine<RM_DP, LPP, LONG, WIDE>,
                         (const void*)k_refine<RM_FIN1, LPP, LONG, WIDE>, (const void*)k_refine<RM_FIN2, LPP, LONG, WIDE>,
                         (const void*)k_refine<RM_PROD1, LPP, LONG, WIDE>, (const void*)k_refine<RM_PROD2, LPP, LONG, WIDE>,
                         (const void*)k_refine<RM_PLOG, LPP, LONG, WIDE>};
    int dev = 0, smem_sm = 0, regs_sm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev);
    cudaDeviceGetAttribute(&regs_sm, cudaDevAttrMaxRegistersPerMultiprocessor, dev);
    for (const void* k : ks) {
        cudaFuncAttributes fa{};
        int carve = 27;
        if (cudaFuncGetAttributes(&fa, k) == cudaSuccess && smem_sm > 0 && fa.numRegs > 0) {
            const int warp_regs = (fa.numRegs * 32 + 255) / 256 * 256;   // per-warp allocation unit
            int ctas = regs_sm / (warp_regs * W);
            if (ctas > 32) ctas = 32;
            const long long need = (long long)ctas * ((long long)fa.sharedSizeBytes + 1024);
            carve = (int)((need * 100 + smem_sm - 1) / smem_sm);
            if (carve < 1) carve = 1;
            if (carve > 100) carve = 100;
        }
        cudaFuncSetAttribute(k, cudaFuncAttributePreferredSharedMemoryCarveout, carve);
    }
}

void configure_kernels() {
    carve_refine<16, false>();
    carve_refine<32, false>();
    carve_refine<32, true>();
    carve_refine<32, true, true>();
    float gs[GTB_GONNET_NA * GTB_GONNET_NA];
    gtb_gonnet_scores(gs);
    cudaMemcpyToSymbol(g_gonnet, gs, sizeof(gs));
}

static void launch_refine_long_fin(int mode, const Blk& B, const Bat& T, cudaStream_t st) {
    const int ng = (T.rl_nlmax + 3) / 4;
    switch (mode) {
        case RM_INIT:  k_refine_long_fin<RM_INIT><<<ng, 128, 0, st>>>(B, T); break;
        case RM_DP:    k_refine_long_fin<RM_DP><<<ng, 128, 0, st>>>(B, T); break;
        case RM_FIN1:  k_refine_long_fin<RM_FIN1><<<ng, 128, 0, st>>>(B, T); break;
        case RM_FIN2:  k_refine_long_fin<RM_FIN2><<<ng, 128, 0, st>>>(B, T); break;
        case RM_PROD1: k_refine_long_fin<RM_PROD1><<<ng, 128, 0, st>>>(B, T); break;
        case RM_PROD2: k_refine_long_fin<RM_PROD2><<<ng, 128, 0, st>>>(B, T); break;
        case RM_PLOG:  k_refine_long_fin<RM_PLOG><<<ng, 128, 0, st>>>(B, T); break;
    }
}

void launch_refine(int mode, const Blk& B, const Bat& T0, cudaStream_t st, bool few) {
    // the long-pair path: from RL_LONG positions with T0.rlw_ctas CTAs; where
    // few pairs take part (the launches after the --pre-score filter) a
    // launch lasts as long as its slowest pair, so there the pairs from
    // RL_LONG_FEW positions below that get RLW_CTAS_FEW CTAs (second tier)
    Bat T = T0;
    T.rl_min = RL_LONG;
    T.rlw_ctas = T0.rlw_ctas > 0 && T0.rlw_ctas <= RLW_CTAS_MAX ? T0.rlw_ctas : RLW_CTAS;
    T.rl_min2 = RL_LONG_FEW;
    T.rlw_ctas2 = T0.rlw_ctas2 > 0 && T0.rlw_ctas2 <= RLW_CTAS_MAX ? T0.rlw_ctas2 : RLW_CTAS_FEW;
    if (!few) T.rl_long2 = nullptr;
    cudaMemsetAsync(T.rhist, 0, (RL_NB + 1) * sizeof(int), st);
    if (T.rl_long) {
        cudaMemsetAsync(T.rl_count, 0, sizeof(int), st);
        cudaMemsetAsync(T.rl_next, 0, (size_t)T.rl_nlmax * sizeof(int), st);
    }
    if (T.rl_long2) {
        cudaMemsetAsync(T.rl_count2, 0, sizeof(int), st);
        cudaMemsetAsync(T.rl_next2, 0, (size_t)T.rl_nlmax2 * sizeof(int), st);
    }
    const int nb = (T.np + 255) / 256;
    k_rlist_count<<<nb, 256, 0, st>>>(B, T, mode);
    k_rlist_scan<<<1, 1024, 0, st>>>(T);
    k_rlist_fill<<<nb, 256, 0, st>>>(B, T, mode);
    // the long pairs on the second stream, beside the short ones (both read
    // the lists built above; they write disjoint pairs)
    const bool fork = T.st2 && (T.rl_long || T.rl_long2);
    cudaStream_t sl = fork ? T.st2 : st;
    KtScope kts(T, KF_REFINE, st);   // on st, after the join: both streams' time
    if (fork) {
        cudaEventRecord(T.evfork, st);
        cudaStreamWaitEvent(T.st2, T.evfork, 0);
    }
    if (few) launch_refine_k<32, false>(mode, B, T, st);
    else launch_refine_k<16, false>(mode, B, T, st);
    if (T.launches) (*T.launches) += 4;
    if (T.rl_long) {
        if (T.rl_nlmax <= RLW_WIDE_MAX) launch_refine_k<32, true, true>(mode, B, T, sl);
        else launch_refine_k<32, true>(mode, B, T, sl);
        launch_refine_long_fin(mode, B, T, sl);
        if (T.launches) (*T.launches) += 2;
    }
    if (T.rl_long2) {
        // the second tier through the same kernels, on its own list
        Bat T2 = T;
        T2.rl_long = T.rl_long2; T2.rl_count = T.rl_count2; T2.rl_next = T.rl_next2;
        T2.rl_cand = T.rl_cand2; T2.rl_nlmax = T.rl_nlmax2; T2.rlw_ctas = T.rlw_ctas2;
        launch_refine_k<32, true>(mode, B, T2, sl);
        launch_refine_long_fin(mode, B, T2, sl);
        if (T.launches) (*T.launches) += 2;
    }
    if (fork) {
        cudaEventRecord(T.evjoin, T.st2);
        cudaStreamWaitEvent(st, T.evjoin, 0);
    }
}

// ---------------------------------------------------------------------------
// DP: MpDPHub.cpp:72-346 and 686-940.  One warp per pair.  Lane l holds the
// R query rows 32*R*s + R*l + r of strip s and, at step t of the strip,
// computes column j = t - l of those rows (one anti-diagonal of the strip
// per step).  The value above a lane's first row comes from lane l-1 (its
// last row, previous step) or, for lane 0, from the previous strip's last
// row kept in `row`.  Stored values are negated when the cell was reached
// diagonally (the reference's state encoding, MpDPHub.cpp:246-262).  Steps
// run in groups of 16/R, one traceback word per lane and group.
// WAVE: the strips of one pair are shared by several CTAs (strip s by CTA
// s mod s_step); a strip waits, with a bounded spin, until the previous one
// has published the steps whose last-row values it is about to read
// (`prog`: steps done per strip), and publishes its own progress every 32
// steps.  Returns false when a wait gave up (error flag set).
// SC, the cell score: DP_SC_TFM (TM-score term under t), DP_SC_TFMSS (plus 0.5
// for equal secondary structure), DP_SC_SSRR (the --add-search-by-ss DP,
// dpssw_btck.cu:280-330: 1 for equal secondary structure + 0.2 x the Gonnet
// score of the residues, no transform; a cell reached diagonally stores its
// value + DPSS_C, a reader takes the offset off again, the gap cost is paid
// once when leaving such a cell; the border reads as a diagonal cell of 0).
// SCOREONLY: no traceback words; the last cell's value goes to *fin.
template <int R, bool gap0, int SC, bool WAVE, bool SCOREONLY = false>
__device__ __forceinline__ bool dp_pair(const float* t, float d02, float gcost, int lq, int lr,
                                        const float* qx, const float* qy, const float* qz,
                                        const float4* r4, const char* qs, const char* rs,
                                        const unsigned char* qa, const unsigned char* ra,
                                        float* row, unsigned* bt, int lane, int s_first = 0,
                                        int s_step = 1, volatile int* prog = nullptr,
                                        volatile int* err = nullptr,
                                        long long spin = DP_WAVE_SPIN_DEFAULT, float* fin = nullptr,
                                        bool cta_wave = false) {
    // cta_wave: the strips' warps share one CTA, so the row values and the
    // progress counters need ordering at CTA scope only
    constexpr bool usess = SC == DP_SC_TFMSS, ssrr = SC == DP_SC_SSRR;
    constexpr float BND = ssrr ? DPSS_C : 0.f;   // the matrix border
    constexpr int ROWS = 32 * R, SPW = 16 / R;
    const unsigned FULL = 0xffffffffu;
    const int W = lr + 31;
    const int ngrp = (W + SPW - 1) / SPW;
    const int nstrips = (lq + ROWS - 1) / ROWS;
    for (int s = s_first; s < nstrips; s += s_step) {
        float tx[R], ty[R], tz[R], h[R];
        char qss[R];
        unsigned char qaa[R];
        int nv = 0;  // valid rows of this lane (a prefix of its R rows)
#pragma unroll
        for (int r = 0; r < R; r++) {
            int irow = s * ROWS + lane * R + r;
            tx[r] = ty[r] = tz[r] = 0.f;
            qss[r] = 0;
            qaa[r] = 0;
            h[r] = BND;
            if (irow < lq) {
                if (!ssrr) xform(t, __ldg(qx + irow), __ldg(qy + irow), __ldg(qz + irow), tx[r], ty[r], tz[r]);
                if (usess || ssrr) qss[r] = qs[irow];
                if (ssrr) qaa[r] = qa[irow];
                nv = r + 1;
            }
        }
        float uplast = BND, rb = BND;
        unsigned* bts = SCOREONLY ? nullptr : bt + (long long)s * ngrp * 32 + lane;
        const bool full = (s + 1) * ROWS <= lq;    // every lane has R rows
        const int lastr = (lq - 1) - s * ROWS - lane * R;   // the last row among this lane's (if 0..R-1)
        __syncwarp();
        for (int g = 0; g < ngrp; g++) {
            unsigned acc = 0u;
            if (WAVE && s > 0 && ((g * SPW) & 31) == 0) {
                // row[tt .. tt+31] of strip s-1: written up to its step tt+62
                const int need = g * SPW + 64 < ngrp * SPW ? g * SPW + 64 : ngrp * SPW;
                if (lane == 0) {
                    long long it = 0;
                    while (prog[s - 1] < need) {
                        if (*err || ++it > spin) { *err = 1; break; }
                        __nanosleep(64);
                    }
                }
                __syncwarp();
                if (cta_wave) __threadfence_block();
                else __threadfence();
                if (*err) return false;
            }
            if ((g * SPW & 31) == 0) {            // the previous strip's last row, 32 columns
                int jj = g * SPW + lane;
                if (WAVE) rb = (s > 0 && jj < lr) ? __ldcg(row + jj) : BND;
                else rb = (s > 0 && jj < lr) ? row[jj] : BND;
            }
            // SPW steps; CHK: some lane may be outside the matrix or have
            // fewer than R rows (strip ramps, the last strip)
            auto steps = [&](auto chk) {
                constexpr bool CHK = decltype(chk)::value;
#pragma unroll
                for (int u = 0; u < SPW; u++) {
                    const int tt = g * SPW + u;   // steps past W find j >= lr on every lane
                    const int j = tt - lane;
                    float upv = __shfl_up_sync(FULL, h[R - 1], 1);
                    float up0 = __shfl_sync(FULL, rb, tt & 31);
                    if (lane == 0) upv = (!CHK || j < lr) ? up0 : BND;
                    if (!CHK || (j >= 0 && j < lr && nv > 0)) {
                        float4 c4 = ssrr ? make_float4(0.f, 0.f, 0.f, 0.f) : __ldg(r4 + j);
                        char css = (usess || ssrr) ? rs[j] : 0;
                        unsigned char cra = ssrr ? ra[j] : 0;
                        float up = upv, dg = uplast;
#pragma unroll
                        for (int r = 0; r < R; r++) {
                            if (ssrr && (!CHK || r < nv)) {
                                float v = __fmaf_rn(gonnet(qaa[r], cra), 0.2f, (float)(qss[r] == css));
                                v = __fadd_rn(v, dg < DPSS_CMP ? __fsub_rn(dg, DPSS_C) : dg);
                                int bk = BT_DIAG;
                                float l = h[r];
                                if (l < DPSS_CMP) l = __fsub_rn(__fadd_rn(gcost, l), DPSS_C);
                                if (v < l) { v = l; bk = BT_LEFT; }
                                float uu = up;
                                if (uu < DPSS_CMP) uu = __fsub_rn(__fadd_rn(gcost, uu), DPSS_C);
                                if (v < uu) { v = uu; bk = BT_UP; }
                                float w = bk == BT_DIAG ? __fadd_rn(v, DPSS_C) : v;
                                dg = h[r];
                                up = w;
                                h[r] = w;
                                acc |= (unsigned)bk << (2 * R * u + 2 * r);
                            } else if (!ssrr && (!CHK || r < nv)) {
                                float v = tmterm(d02, dist2(tx[r], ty[r], tz[r], c4.x, c4.y, c4.z));
                                if (usess) v = __fadd_rn(v, __fmul_rn((float)(qss[r] == css), 0.5f));
                                v = __fadd_rn(v, gap0 ? dg : fabsf(dg));
                                int bk = BT_DIAG;
                                float l = h[r];
                                if (!gap0 && l < 0.f) l = __fsub_rn(gcost, l);
                                if (v < l) { v = l; bk = BT_LEFT; }
                                float uu = up;
                                if (!gap0 && uu < 0.f) uu = __fsub_rn(gcost, uu);
                                if (v < uu) { v = uu; bk = BT_UP; }
                                float w = (gap0 || bk != BT_DIAG) ? v : -v;
                                dg = h[r];   // (row r, j-1): the next row's diagonal
                                up = w;      // (row r, j):   the next row's up
                                h[r] = w;
                                if (SCOREONLY) { if (r == lastr && j == lr - 1) *fin = w; }
                                else acc |= (unsigned)bk << (2 * R * u + 2 * r);
                            }
                        }
                        if (lane == 31 && (!CHK || nv == R)) row[j] = h[R - 1];
                    }
                    uplast = upv;
                }
            };
            if (full && g * SPW >= 31 && (g + 1) * SPW <= lr) steps(std::false_type{});
            else steps(std::true_type{});
            if (!SCOREONLY) bts[g * 32] = acc;
            // the next strip reads its row values 32 steps at a time, so the
            // count is published at every 32nd step (and the last): one fence
            // per 32 steps instead of per group
            if (WAVE && lane == 31 && ((((g + 1) * SPW) & 31) == 0 || g == ngrp - 1)) {
                if (cta_wave) __threadfence_block();   // the row values before the count
                else __threadfence();
                prog[s] = (g + 1) * SPW;
            }
        }
        __syncwarp();
    }
    return true;
}

// The DP work list (k_dlist_*, largest matrices first): its first dp_kc
// pairs take a CTA each, whose 4 warps run the pair's strips as a wavefront
// (strip s on warp s mod 4, each strip waiting with a bounded spin until the
// previous one has published the row values it reads, the counters in
// shared memory); the other pairs take a warp each.
template <int GAP0, int SC>
__global__ void __launch_bounds__(128) k_dp(Blk B, Bat T, int tfmsrc, float gcost, int dpscan,
                                            int skipmode) {
    __shared__ int s_prog[DP_CTA_MAXSTRIPS];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int len = T.rhist[RL_NB];
    const int dkc = T.dw_err ? T.dp_kc : 0;
    const int kc = dkc < len ? dkc : len;
    const bool cta = (int)blockIdx.x < kc;
    const int slot = cta ? (int)blockIdx.x : kc + ((int)blockIdx.x - kc) * (blockDim.x >> 5) + w;
    if (slot >= len) return;                       // never for a CTA of the first kind
    const int i = T.rlist[slot];
    int qi = pair_qi(B, T, i), ri = pair_ri(B, T, i);
    int lq = B.qlen[qi], lr = B.rlen[ri];
    int ml = lq < lr ? lq : lr;
    const float* tsrc = dp_tfm(T, i, tfmsrc);
    float t[12];
#pragma unroll
    for (int f = 0; f < 12; f++) t[f] = tsrc[f];
    float d0 = B.t_d0[ml];
    float d02;
    if (dpscan) { float a = __fadd_rn(d0, 1.5f); d02 = __fmul_rn(a, a); }
    else d02 = __fmul_rn(d0, d0);
    const float* qx = B.qx + B.qoff[qi];
    const float* qy = B.qy + B.qoff[qi];
    const float* qz = B.qz + B.qoff[qi];
    const float4* r4 = B.r4 + B.r4off[ri];
    const char* qs = B.qs + B.qoff[qi];
    const char* rs = B.rs + B.roff[ri];
    float* row = T.row + T.off_row[i];
    unsigned* bt = T.bt + T.off_bt[i];
    const unsigned char* qa = B.qa + B.qoff[qi];
    const unsigned char* ra = B.ra + B.roff[ri];
    if (cta) {
        if (lane == 0 && w == 0) work_add(T, WK_DPCELL, (unsigned long long)lq * (unsigned long long)lr);
        if (dp_strips(lq) > 1) {
            for (int k = threadIdx.x; k < DP_CTA_MAXSTRIPS; k += blockDim.x) s_prog[k] = 0;
            __syncthreads();
            if (dp_r(lq) == 4)
                dp_pair<4, GAP0 != 0, SC, true>(t, d02, gcost, lq, lr, qx, qy, qz, r4, qs, rs, qa, ra, row,
                                                bt, lane, w, blockDim.x >> 5, s_prog, T.dw_err, T.dw_spin,
                                                nullptr, true);
            else
                dp_pair<2, GAP0 != 0, SC, true>(t, d02, gcost, lq, lr, qx, qy, qz, r4, qs, rs, qa, ra, row,
                                                bt, lane, w, blockDim.x >> 5, s_prog, T.dw_err, T.dw_spin,
                                                nullptr, true);
            return;
        }
        if (w != 0) return;                        // one strip: one warp
    } else if (lane == 0) {
        work_add(T, WK_DPCELL, (unsigned long long)lq * (unsigned long long)lr);
    }
    if (dp_r(lq) == 4)
        dp_pair<4, GAP0 != 0, SC, false>(t, d02, gcost, lq, lr, qx, qy, qz, r4, qs, rs, qa, ra, row, bt, lane);
    else
        dp_pair<2, GAP0 != 0, SC, false>(t, d02, gcost, lq, lr, qx, qy, qz, r4, qs, rs, qa, ra, row, bt, lane);
}

// One warp per CTA; the CTAs of a long pair take its strips round robin.
// Launched cooperatively so that all CTAs are resident together.
template <int GAP0, int SC>
__global__ void __launch_bounds__(32) k_dp_wave(Blk B, Bat T, int tfmsrc, float gcost, int dpscan,
                                                int skipmode) {
    const int lane = threadIdx.x & 31;
    const int item = blockIdx.x;
    if (item >= T.ndw) return;
    const int slot = T.dw_item[item], c = T.dw_item[T.ndw + item];
    const int i = T.dw_pair[slot], G = T.dw_G[slot];
    int flags = T.flags[i];
    int skipmask = skipmode == 0 ? (CONV_LOWTMSC | CONV_SCOREDP) : CONV_LOWTMSC;
    if (flags & skipmask) return;                  // the same for every CTA of the pair
    if (alt_empty(T, i)) return;
    int qi = pair_qi(B, T, i), ri = pair_ri(B, T, i);
    int lq = B.qlen[qi], lr = B.rlen[ri];
    int ml = lq < lr ? lq : lr;
    const float* tsrc = dp_tfm(T, i, tfmsrc);
    float t[12];
#pragma unroll
    for (int f = 0; f < 12; f++) t[f] = tsrc[f];
    float d0 = B.t_d0[ml];
    float d02;
    if (dpscan) { float a = __fadd_rn(d0, 1.5f); d02 = __fmul_rn(a, a); }
    else d02 = __fmul_rn(d0, d0);
    const float* qx = B.qx + B.qoff[qi];
    const float* qy = B.qy + B.qoff[qi];
    const float* qz = B.qz + B.qoff[qi];
    const float4* r4 = B.r4 + B.r4off[ri];
    const char* qs = B.qs + B.qoff[qi];
    const char* rs = B.rs + B.roff[ri];
    float* row = T.row + T.off_row[i];
    unsigned* bt = T.bt + T.off_bt[i];
    volatile int* prog = T.dw_prog + T.dw_soff[slot];
    const unsigned char* qa = B.qa + B.qoff[qi];
    const unsigned char* ra = B.ra + B.roff[ri];
    if (lane == 0 && c == 0) work_add(T, WK_DPCELL, (unsigned long long)lq * (unsigned long long)lr);
    if (dp_r(lq) == 4)
        dp_pair<4, GAP0 != 0, SC, true>(t, d02, gcost, lq, lr, qx, qy, qz, r4, qs, rs, qa, ra, row,
                                        bt, lane, c, G, prog, T.dw_err, T.dw_spin);
    else
        dp_pair<2, GAP0 != 0, SC, true>(t, d02, gcost, lq, lr, qx, qy, qz, r4, qs, rs, qa, ra, row,
                                        bt, lane, c, G, prog, T.dw_err, T.dw_spin);
}

int dp_wave_capacity() {
    int dev = 0, nsm = 0, m = 1 << 30, nb = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    const void* ks[5] = {(const void*)k_dp_wave<1, DP_SC_TFM>, (const void*)k_dp_wave<0, DP_SC_TFM>,
                         (const void*)k_dp_wave<0, DP_SC_TFMSS>, (const void*)k_dp_wave<1, DP_SC_TFMSS>,
                         (const void*)k_dp_wave<0, DP_SC_SSRR>};
    for (const void* k : ks) {
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k, 32, 0) != cudaSuccess) return 0;
        m = nb < m ? nb : m;
    }
    return m * nsm;
}

template <int GAP0, int SC>
static void launch_dp_wave(const Blk& B, const Bat& T, int tfmsrc, float gcost, int dpscan,
                           int skipmode, cudaStream_t st) {
    Blk b = B;
    Bat t = T;
    void* args[] = {&b, &t, &tfmsrc, &gcost, &dpscan, &skipmode};
    cudaError_t e = cudaLaunchCooperativeKernel((const void*)k_dp_wave<GAP0, SC>, dim3(T.ndw),
                                                dim3(32), args, 0, st);
    if (e != cudaSuccess && T.lerr && *T.lerr == cudaSuccess) *T.lerr = e;
}

void launch_dp(const Blk& B, const Bat& T, int tfmsrc, int gap0, float gcost, int usess,
               int dpscan, int skipmode, cudaStream_t st) {
    {
        cudaMemsetAsync(T.rhist, 0, (RL_NB + 1) * sizeof(int), st);
        const int nb = (T.np + 255) / 256;
        k_dlist_count<<<nb, 256, 0, st>>>(B, T, skipmode);
        k_rlist_scan<<<1, 1024, 0, st>>>(T);
        k_dlist_fill<<<nb, 256, 0, st>>>(B, T, skipmode);
        if (T.launches) (*T.launches) += 3;
    }
    KtScope kts(T, KF_DP, st);
    if (T.ndw > 0) {
        cudaMemsetAsync(T.dw_prog, 0, (size_t)T.dw_nprog * sizeof(int), st);
        if (usess == DP_SC_SSRR) launch_dp_wave<0, DP_SC_SSRR>(B, T, tfmsrc, gcost, dpscan, skipmode, st);
        else if (gap0 && !usess) launch_dp_wave<1, DP_SC_TFM>(B, T, tfmsrc, gcost, dpscan, skipmode, st);
        else if (!gap0 && !usess) launch_dp_wave<0, DP_SC_TFM>(B, T, tfmsrc, gcost, dpscan, skipmode, st);
        else if (!gap0 && usess) launch_dp_wave<0, DP_SC_TFMSS>(B, T, tfmsrc, gcost, dpscan, skipmode, st);
        else launch_dp_wave<1, DP_SC_TFMSS>(B, T, tfmsrc, gcost, dpscan, skipmode, st);
        GTB_LAUNCHED(T);
    }
    // dp_kc CTAs for the largest listed pairs, then a warp per pair
    const int nb = (T.dw_err ? T.dp_kc : 0) + (T.np + 3) / 4;
    if (usess == DP_SC_SSRR) k_dp<0, DP_SC_SSRR><<<nb, 128, 0, st>>>(B, T, tfmsrc, gcost, dpscan, skipmode);
    else if (gap0 && !usess) k_dp<1, DP_SC_TFM><<<nb, 128, 0, st>>>(B, T, tfmsrc, gcost, dpscan, skipmode);
    else if (!gap0 && !usess) k_dp<0, DP_SC_TFM><<<nb, 128, 0, st>>>(B, T, tfmsrc, gcost, dpscan, skipmode);
    else if (!gap0 && usess) k_dp<0, DP_SC_TFMSS><<<nb, 128, 0, st>>>(B, T, tfmsrc, gcost, dpscan, skipmode);
    else k_dp<1, DP_SC_TFMSS><<<nb, 128, 0, st>>>(B, T, tfmsrc, gcost, dpscan, skipmode);
    GTB_LAUNCHED(T);
}

void launch_pair_list(const Blk& B, const Bat& T, int skipmask, cudaStream_t st) {
    cudaMemsetAsync(T.rhist, 0, (RL_NB + 1) * sizeof(int), st);
    const int nb = (T.np + 255) / 256;
    k_plist_count<<<nb, 256, 0, st>>>(B, T, skipmask);
    k_rlist_scan<<<1, 1024, 0, st>>>(T);
    k_plist_fill<<<nb, 256, 0, st>>>(B, T, skipmask);
    if (T.launches) (*T.launches) += 3;
}

// Detailed search: the DP scores of a pair's fragment slots
// (ExecDPScore128xKernel, MpDPHub.cpp:389-645): for every slot with a
// positive score, the last cell of the gap-0 DP under the slot's transform
// (search d0), no traceback; 0 for the others.  A warp per (listed pair,
// slot) item, the items walked by a grid of resident warps in list order
// (largest pairs first); each slot's DP keeps its strip row in the pair's
// detailed-search region (the local score matrix is no longer read).
__global__ void __launch_bounds__(128) k_f3_dpscore(Blk B, Bat T) {
    const int lane = threadIdx.x & 31;
    const int nsl = B.f3nsec * F3_NTOP;          // slots per pair
    const long long nitems = (long long)T.rhist[RL_NB] * nsl;
    const long long wstride = (long long)gridDim.x * (blockDim.x >> 5);
    for (long long it = (long long)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); it < nitems;
         it += wstride) {
        const int i = T.rlist[it / nsl];
        const int k = (int)(it % nsl);
        const float* sl = T.f3slot + ((long long)i * nsl + k) * 13;
        float* fin = T.f3dps + (long long)i * nsl + k;
        if (!(0.f < sl[0])) {
            if (lane == 0) *fin = 0.f;
            continue;
        }
        int qi = pair_qi(B, T, i), ri = pair_ri(B, T, i);
        int lq = B.qlen[qi], lr = B.rlen[ri];
        int ml = lq < lr ? lq : lr;
        const float d0 = B.t_d0[ml];
        const float d02 = __fmul_rn(d0, d0);
        const float* qx = B.qx + B.qoff[qi];
        const float* qy = B.qy + B.qoff[qi];
        const float* qz = B.qz + B.qoff[qi];
        const float4* r4 = B.r4 + B.r4off[ri];
        float* row = (float*)(T.lsm + T.off_lsm[i]) + (long long)k * lr;
        float t[12];
#pragma unroll
        for (int f = 0; f < 12; f++) t[f] = sl[1 + f];
        if (lane == 0) work_add(T, WK_F3CELL, (unsigned long long)lq * (unsigned long long)lr);
        if (dp_r(lq) == 4)
            dp_pair<4, true, DP_SC_TFM, false, true>(t, d02, 0.f, lq, lr, qx, qy, qz, r4, nullptr,
                                                     nullptr, nullptr, nullptr, row, nullptr, lane,
                                                     0, 1, nullptr, nullptr, DP_WAVE_SPIN_DEFAULT, fin);
        else
            dp_pair<2, true, DP_SC_TFM, false, true>(t, d02, 0.f, lq, lr, qx, qy, qz, r4, nullptr,
                                                     nullptr, nullptr, nullptr, row, nullptr, lane,
                                                     0, 1, nullptr, nullptr, DP_WAVE_SPIN_DEFAULT, fin);
        __syncwarp();
    }
}

void launch_f3_dpscore(const Blk& B, const Bat& T, cudaStream_t st) {
    // enough warps to fill the GPU (the kernel walks its items)
    int dev = 0, nsm = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    const long long need = ((long long)T.np * B.f3nsec * F3_NTOP + 3) / 4;
    const int ng = (int)std::min<long long>(need, (long long)nsm * 8);
    k_f3_dpscore<<<ng > 0 ? ng : 1, 128, 0, st>>>(B, T);
    GTB_LAUNCHED(T);
}

// ---------------------------------------------------------------------------
// traceback: MpDPHub.cpp:1515-1660 (plain) and 1699-1905 (constrained)
constexpr int BTCK_AHEAD = 4;     // step groups the traceback loads ahead
__device__ __forceinline__ void bt_prefetch(const unsigned* p) {
    asm volatile("prefetch.global.L1 [%0];" ::"l"(p));
}

__global__ void k_btck(Blk B, Bat T, int constrained) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= T.np) return;
    int flags = T.flags[i];
    if (constrained) {
        if (flags & CONV_LOWTMSC) return;
    } else if ((flags & (CONV_LOWTMSC | CONV_SCOREDP)) || alt_empty(T, i)) {
        T.naln[i] = 0;
        return;
    }
    int qi = pair_qi(B, T, i), ri = pair_ri(B, T, i);
    int lq = B.qlen[qi], lr = B.rlen[ri];
    int ml = lq < lr ? lq : lr;
    const unsigned* bt = T.bt + T.off_bt[i];
    unsigned* aln = T.aln + T.off_aln[i];
    float* alc = T.alc + 6 * T.off_aln[i];
    const int R = dp_r(lq), rows = 32 * R, spw = 16 / R;
    const long long sw = bt_strip_words(lr, R);
    float t[12];
    float d82 = B.t_d82[ml];
    const float4* q4 = B.q4 + B.q4off[qi];
    const float4* r4 = B.r4 + B.r4off[ri];
    if (constrained) {
#pragma unroll
        for (int f = 0; f < 12; f++) t[f] = T.tfm_gr[i * 12 + f];
    }
    int y = lq - 1, x = lr - 1, n = 0;
    // The walk is a chain of dependent loads.  The 32 words of a (strip, step
    // group) are one 128-byte line and the path only moves to lower groups and
    // strips, so each new group starts the loads of the BTCK_AHEAD groups
    // below it (and, near a strip's top, of the previous strip's groups the
    // path enters next); the last word read is kept.
    long long cwi = -1;
    unsigned w = 0;
    int cs = -1, cg = -1, prevs = -1;
    while (x >= 0 && y >= 0) {
        int yy = y % rows, l = yy / R, tt = x + l;
        const int s = y / rows, g = tt / spw;
        const long long wi = (long long)s * sw + (long long)g * 32 + l;
        if (wi != cwi) {
            if (s != cs) {              // a new strip (or the start): its next groups
                for (int k = 1; k <= BTCK_AHEAD && g - k >= 0; k++)
                    bt_prefetch(bt + (long long)s * sw + (long long)(g - k) * 32);
            } else if (g != cg && g >= BTCK_AHEAD) {
                bt_prefetch(bt + (long long)s * sw + (long long)(g - BTCK_AHEAD) * 32);
            }
            cs = s; cg = g;
            if (l <= 2 && s > 0 && prevs != s) {
                const int gp = (x + 31) / spw;
                for (int k = 0; k < BTCK_AHEAD && gp - k >= 0; k++)
                    bt_prefetch(bt + (long long)(s - 1) * sw + (long long)(gp - k) * 32);
                prevs = s;
            }
            w = bt[wi];
            cwi = wi;
        }
        int b = (int)((w >> (2 * R * (tt % spw) + 2 * (yy % R))) & 3u);
        if (b == BT_UP) { y--; continue; }
        if (b == BT_LEFT) { x--; continue; }
        float4 cq = __ldg(q4 + y), cr = __ldg(r4 + x);
        float cqx = cq.x, cqy = cq.y, cqz = cq.z, crx = cr.x, cry = cr.y, crz = cr.z;
        bool keep = true;
        if (constrained) keep = dist2_tf(t, cqx, cqy, cqz, crx, cry, crz) <= d82;
        if (keep) {
            aln[n] = ((unsigned)y << 16) | (unsigned)x;
            float2* c2 = (float2*)(alc + 6 * (long long)n);
            c2[0] = make_float2(cqx, cqy); c2[1] = make_float2(cqz, crx); c2[2] = make_float2(cry, crz);
            n++;
        }
        x--; y--;
    }
    T.naln[i] = n;
}

void launch_btck(const Blk& B, const Bat& T, int constrained, cudaStream_t st) {
    k_btck<<<(T.np + 127) / 128, 128, 0, st>>>(B, T, constrained);
    GTB_LAUNCHED(T);
}

// ---------------------------------------------------------------------------
// per-iteration bookkeeping of DPRefine: MpStage1.cpp:495-513 and
// CheckScoreConvergence / SaveLastScore0 / SetLowScoreConvergenceFlag
__global__ void k_post(Blk B, Bat T, int dpi, int maxit, int prescreen, float prescore) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= T.np) return;
    int flags = T.flags[i];
    float best = T.best[i];
    if (0 < dpi && !(flags & (CONV_SCOREDP | CONV_LOWTMSC)) &&
        fabsf(__fsub_rn(best, T.best0[i])) < SCORE_CONVEPS)
        flags |= CONV_SCOREDP;
    if (dpi + 1 < maxit && !(flags & (CONV_SCOREDP | CONV_LOWTMSC)))
        T.best0[i] = best;
    if (prescreen && maxit <= dpi + 1 && 0.0f < prescore) {
        int qi = pair_qi(B, T, i), ri = pair_ri(B, T, i);
        int lq = B.qlen[qi], lr = B.rlen[ri];
        int ml = lq < lr ? lq : lr;
        if (T.grand[i] < __fmul_rn(prescore, (float)ml)) flags |= CONV_LOWTMSC;
    }
    if (dpi == maxit - 1) flags &= ~CONV_SCOREDP;
    T.flags[i] = flags;
}

void launch_post(const Blk& B, const Bat& T, int dpi, int maxit, int prescreen, float prescore,
                 cudaStream_t st) {
    k_post<<<(T.np + 255) / 256, 256, 0, st>>>(B, T, dpi, maxit, prescreen, prescore);
    GTB_LAUNCHED(T);
}

__global__ void k_lowscore(Blk B, Bat T, float thr) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= T.np) return;
    int qi = pair_qi(B, T, i), ri = pair_ri(B, T, i);
    int lq = B.qlen[qi], lr = B.rlen[ri];
    int ml = lq < lr ? lq : lr;
    if (T.grand[i] < __fmul_rn(thr, (float)ml)) T.flags[i] |= CONV_LOWTMSC;
}

void launch_lowscore(const Blk& B, const Bat& T, float thr, cudaStream_t st) {
    k_lowscore<<<(T.np + 255) / 256, 256, 0, st>>>(B, T, thr);
    GTB_LAUNCHED(T);
}

// ---------------------------------------------------------------------------
// alignment rows: MpDPHub.cpp:1919-2125.  The rows of a pair with an
// alignment are packed at an offset it reserves (atomically) once its column
// count is known; that count follows from the first and last aligned pairs:
// every aligned pair is one column, every skipped query residue between them
// one, and every skipped reference residue one unless --no-deletions.
__global__ void k_alnstr(Blk B, Bat T) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= T.np) return;
    if (T.flags[i] & CONV_LOWTMSC) {
        if (T.str) T.str_off[i] = -1;      // no alignment
        return;
    }
    int qi = pair_qi(B, T, i), ri = pair_ri(B, T, i);
    const unsigned* aln = T.aln + T.off_aln[i];
    int n = T.naln[i];
    float t[12];
#pragma unroll
    for (int f = 0; f < 12; f++) t[f] = T.tfm_gr[i * 12 + f];
    const float *qx = B.qx + B.qoff[qi], *qy = B.qy + B.qoff[qi], *qz = B.qz + B.qoff[qi];
    const float *rx = B.rx + B.roff[ri], *ry = B.ry + B.roff[ri], *rz = B.rz + B.roff[ri];
    const unsigned char* qa = B.qa + B.qoff[qi];
    const unsigned char* ra = B.ra + B.roff[ri];
    const char* qs = B.qs + B.qoff[qi];
    const char* rs = B.rs + B.roff[ri];
    char* dst = nullptr;
    int W = 1;
    if (T.str) {
        int ncol = 0;
        if (n > 0) {
            const unsigned wf = aln[n - 1], wl = aln[0];   // first and last aligned pairs
            const int qf = (int)(wf >> 16), rf = (int)(wf & 0xffffu);
            const int ql = (int)(wl >> 16), rl = (int)(wl & 0xffffu);
            ncol = n + (ql - qf + 1 - n) + (B.nodeletions ? 0 : (rl - rf + 1 - n));
        }
        W = ncol + 1;
        const unsigned long long o = atomicAdd(T.str_cnt, 5ull * (unsigned long long)W);
        T.str_off[i] = (long long)o;
        dst = T.str + o;
    }
    int col = 0, psts = 0, idts = 0, gaps = 0;
    unsigned bc = 0, ec = 0;
    for (int k = 0; k < n; k++) {
        unsigned wv = aln[n - 1 - k];
        int q = (int)(wv >> 16), r = (int)(wv & 0xffffu);
        float d = dist2_tf(t, qx[q], qy[q], qz[q], rx[r], ry[r], rz[r]);
        unsigned cc = ((unsigned)(r + 1) << 16) | (unsigned)(q + 1);
        if (k == 0) bc = cc;
        ec = cc;
        int eq = d < 25.0f;
        if (eq) psts++;
        char a = (char)qa[q], b = (char)ra[r];
        char mc = eq ? '+' : ' ';
        if (a != '-' && a == b) { idts++; mc = eq ? a : (char)(a | 32); }
        if (dst) { dst[col] = a; dst[2 * W + col] = b; dst[3 * W + col] = qs[q]; dst[4 * W + col] = rs[r]; dst[W + col] = mc; }
        col++;
        if (k + 1 < n) {
            unsigned w1 = aln[n - 2 - k];
            int q1 = (int)(w1 >> 16), r1 = (int)(w1 & 0xffffu);
            for (int qq = q + 1; qq < q1; qq++) {
                if (dst) { dst[col] = (char)qa[qq]; dst[3 * W + col] = qs[qq]; dst[2 * W + col] = '-'; dst[4 * W + col] = ' '; dst[W + col] = ' '; }
                col++; gaps++;
            }
            if (!B.nodeletions)
                for (int rr = r + 1; rr < r1; rr++) {
                    if (dst) { dst[2 * W + col] = (char)ra[rr]; dst[4 * W + col] = rs[rr]; dst[col] = '-'; dst[3 * W + col] = ' '; dst[W + col] = ' '; }
                    col++; gaps++;
                }
        }
    }
    if (dst) { dst[col] = 0; dst[W + col] = 0; dst[2 * W + col] = 0; dst[3 * W + col] = 0; dst[4 * W + col] = 0; }
    T.out[i * 16 + 2] = __uint_as_float(bc);
    T.out[i * 16 + 3] = __uint_as_float(ec);
    T.out[i * 16 + 4] = (float)col;
    T.out[i * 16 + 5] = (float)psts;
    T.out[i * 16 + 6] = (float)idts;
    T.out[i * 16 + 7] = (float)gaps;
}

void launch_alnstr(const Blk& B, const Bat& T, cudaStream_t st) {
    k_alnstr<<<(T.np + 127) / 128, 128, 0, st>>>(B, T);
    GTB_LAUNCHED(T);
}

// ---------------------------------------------------------------------------
// FP64 recomputation of the reported TM-scores and RMSD, --referenced
__global__ void k_final(Blk B, Bat T, int referenced) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= T.np) return;
    if (T.flags[i] & CONV_LOWTMSC) return;
    int qi = pair_qi(B, T, i), ri = pair_ri(B, T, i);
    int lq = B.qlen[qi], lr = B.rlen[ri];
    const unsigned* aln = T.aln + T.off_aln[i];
    int n = T.naln[i];
    float* t = T.tfm_gr + i * 12;
    float* out = T.out + i * 16;
    if (n > 0) {
        const float *qx = B.qx + B.qoff[qi], *qy = B.qy + B.qoff[qi], *qz = B.qz + B.qoff[qi];
        const float *rx = B.rx + B.roff[ri], *ry = B.ry + B.roff[ri], *rz = B.rz + B.roff[ri];
        const char *qs = B.qs + B.qoff[qi], *rs = B.rs + B.roff[ri];
        double d0q = (double)B.t_d0fin[lq], d0r = (double)B.t_d0fin[lr];
        double d0q2 = __dmul_rn(d0q, d0q), d0r2 = __dmul_rn(d0r, d0r), tq = 0.0, tr = 0.0;
        double t2q = 0.0, t2r = 0.0;   // --2tm-score sums
        double dv[21];
#pragma unroll
        for (int f = 0; f < 21; f++) dv[f] = 0.0;
        double td[12];
#pragma unroll
        for (int f = 0; f < 12; f++) td[f] = (double)t[f];
        for (int k = 0; k < n; k++) {
            unsigned wv = aln[n - 1 - k];
            int q = (int)(wv >> 16), r = (int)(wv & 0xffffu);
            double qq[3] = {(double)qx[q], (double)qy[q], (double)qz[q]};
            double rr[3] = {(double)rx[r], (double)ry[r], (double)rz[r]};
            double x = __dadd_rn(__dadd_rn(__dadd_rn(__dmul_rn(td[0], qq[0]), __dmul_rn(td[1], qq[1])), __dmul_rn(td[2], qq[2])), td[9]);
            double y = __dadd_rn(__dadd_rn(__dadd_rn(__dmul_rn(td[3], qq[0]), __dmul_rn(td[4], qq[1])), __dmul_rn(td[5], qq[2])), td[10]);
            double z = __dadd_rn(__dadd_rn(__dadd_rn(__dmul_rn(td[6], qq[0]), __dmul_rn(td[7], qq[1])), __dmul_rn(td[8], qq[2])), td[11]);
            double dx = __dsub_rn(x, rr[0]), dy = __dsub_rn(y, rr[1]), dz = __dsub_rn(z, rr[2]);
            double d = __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz));
            const double sq = __ddiv_rn(d0q2, __dadd_rn(d0q2, d));
            const double sr = __ddiv_rn(d0r2, __dadd_rn(d0r2, d));
            tq = __dadd_rn(tq, sq);
            tr = __dadd_rn(tr, sr);
            if (B.twotm) {
                // MpStageBase.h:825-856: a helix aligned to a non-helix residue is left out
                const char a2 = qs[q], b2 = rs[r];
                if (!((a2 == 'h' || b2 == 'h') && a2 != b2)) { t2q = __dadd_rn(t2q, sq); t2r = __dadd_rn(t2r, sr); }
            }
#pragma unroll
            for (int a = 0; a < 3; a++)
#pragma unroll
                for (int b = 0; b < 3; b++) dv[3 * a + b] = __dadd_rn(dv[3 * a + b], __dmul_rn(qq[a], rr[b]));
#pragma unroll
            for (int a = 0; a < 3; a++) {
                dv[9 + a] = __dadd_rn(dv[9 + a], qq[a]);
                dv[12 + a] = __dadd_rn(dv[12 + a], rr[a]);
                dv[15 + a] = __dadd_rn(dv[15 + a], __dmul_rn(qq[a], qq[a]));
                dv[18 + a] = __dadd_rn(dv[18 + a], __dmul_rn(rr[a], rr[a]));
            }
        }
        double r64 = rmsd_from_sums(dv, (double)n);
        float r32 = T.rmsd32[i];
        if (r32 >= 0.f) {
            T.err[i * 4 + 2] = (float)fabs(__dsub_rn((double)r32, r64));
            out[8] = (float)r64;
        }
        if (out[9] > 0.f || out[10] > 0.f) {
            double tmq = __ddiv_rn(tq, (double)lq), tmr = __ddiv_rn(tr, (double)lr);
            T.err[i * 4 + 0] = (float)fabs(__dsub_rn((double)out[9], tmq));
            T.err[i * 4 + 1] = (float)fabs(__dsub_rn((double)out[10], tmr));
            out[9] = (float)tmq;
            out[10] = (float)tmr;
        }
        if (B.twotm) {
            // secondary TM-scores (MpStageFin.cpp:1723-1818), FP64 like the primary ones
            out[13] = (float)__ddiv_rn(t2q, (double)lq);
            out[14] = (float)__ddiv_rn(t2r, (double)lr);
        }
    }
    if (referenced) {
        float R[9];
#pragma unroll
        for (int f = 0; f < 9; f++) R[f] = t[f];
#pragma unroll
        for (int a = 0; a < 3; a++)
#pragma unroll
            for (int b = 0; b < 3; b++) t[3 * a + b] = R[3 * b + a];
        float t0 = t[9], t1 = t[10], t2 = t[11];
        t[9] = -__fadd_rn(__fadd_rn(__fmul_rn(R[0], t0), __fmul_rn(R[3], t1)), __fmul_rn(R[6], t2));
        t[10] = -__fadd_rn(__fadd_rn(__fmul_rn(R[1], t0), __fmul_rn(R[4], t1)), __fmul_rn(R[7], t2));
        t[11] = -__fadd_rn(__fadd_rn(__fmul_rn(R[2], t0), __fmul_rn(R[5], t1)), __fmul_rn(R[8], t2));
    }
}

void launch_final(const Blk& B, const Bat& T, int referenced, cudaStream_t st) {
    k_final<<<(T.np + 127) / 128, 128, 0, st>>>(B, T, referenced);
    GTB_LAUNCHED(T);
}

// ---------------------------------------------------------------------------
// Per-length constants; the FP32 formulas of stagecnsts.cuh:48-175 (host).
void make_tables(float* d0, float* d82, float* d0fin, int n) {
    for (int L = 0; L < n; L++) {
        float l = (float)L;
        float a = 0.168f;
        if (l > 19.f) a = 1.24f * cbrtf(l - 15.f) - 1.8f;
        d0[L] = a + 0.8f;
        float d8 = 1.5f * powf(l, 0.3f) + 3.5f;
        d82[L] = d8 * d8;
        float f = 0.5f;
        if (l > 21.f) f = 1.24f * cbrtf(l - 15.f) - 1.8f;
        if (f < 0.5f) f = 0.5f;
        d0fin[L] = f;
    }
}

// DPRefine (MpStage1.cpp:466-517): maxit rounds of DP, traceback, fragment
// refinement over the alignment and the convergence bookkeeping; the first
// DP uses the transform tfm1 (DP_TFM_IBEST, or DP_TFM_2ND after the detailed
// search, WRKMEMTM1)
void launch_dprefine(const Blk& B, const Bat& T, int gap0, int prescreen, int maxit,
                     float prescore, bool few, int tfm1, cudaStream_t st) {
    for (int dpi = 0; dpi < maxit; dpi++) {
        launch_dp(B, T, dpi == 0 ? tfm1 : DP_TFM_IBEST, gap0, gap0 ? 0.0f : -0.6f, 0, 0, 0, st);
        launch_btck(B, T, 0, st);
        launch_refine(RM_DP, B, T, st, few);
        launch_post(B, T, dpi, maxit, prescreen, prescore, st);
    }
}

// ---------------------------------------------------------------------------
// The stage sequence of one batch: CuBatch::ProcessBlock (CuBatch.cu:537-700)
// with the detailed search off.  ev (may be null): 5 events recorded at the
// stage boundaries.
void launch_stages(const Blk& B, const Bat& T, int refinement, int depth, int convergence,
                   float prescore, int referenced, float scorethld, cudaStream_t st,
                   cudaEvent_t* ev, int polish_steps) {
    auto mark = [&](int k) { if (ev) cudaEventRecord(ev[k], st); };
    // DPRefine: MpStage1.cpp:466-517
    // after the stage-1 --pre-score filter only a small share of pairs is left
    const bool few = 0.0f < prescore;
    auto dprefine = [&](int gap0, int prescreen, int maxit, bool fewp) {
        launch_dprefine(B, T, gap0, prescreen, maxit, prescore, fewp, DP_TFM_IBEST, st);
    };
    mark(0);
    launch_init(B, T, st);
    if (B.presim > 0.f) launch_presim(B, T, st);
    launch_findfrag(B, T, st);
    mark(1);
    launch_refine(RM_INIT, B, T, st, false);
    mark(2);
    dprefine(1, 1, 2, false);
    if (B.addss) {
        // --add-search-by-ss (custage_ssrr.cu:43-140, CuBatch.cu:583-600): the
        // alignment of the SS and residue-scored DP, fragment refinement over it,
        // DP refinement with the gap cost and without, 2 iterations each
        launch_dp(B, T, DP_TFM_GRAND, 0, -1.0f, DP_SC_SSRR, 0, 1, st);
        launch_btck(B, T, 0, st);
        launch_refine(RM_DP, B, T, st, few);
        dprefine(0, 0, 2, few);
        dprefine(1, 0, 2, few);
    }
    // the spatial-index detailed search (CuBatch.cu:612-623)
    if (B.f3) launch_frg3(B, T, st);
    // two stage-2 passes: MpStage2.h:63-83, CuBatch.cu:627-650
    for (int call = 0; call < 2; call++) {
        int gap0 = call == 1;
        launch_dp(B, T, DP_TFM_GRAND, gap0, gap0 ? 0.0f : -1.0f, !gap0, !gap0, 1, st);
        launch_btck(B, T, 0, st);
        launch_refine(RM_DP, B, T, st, few);
        dprefine(0, 0, 2, few);
        dprefine(1, 0, call == 0 ? 2 : convergence, few);
        if (call == 1 && 0.0f < scorethld) launch_lowscore(B, T, scorethld, st);
    }
    mark(3);
    // final stage: MpStageFin.h:63-96
    launch_dp(B, T, DP_TFM_GRAND, 1, 0.0f, 0, 0, 1, st);
    launch_btck(B, T, 0, st);
    launch_refine(RM_FIN1, B, T, st, few);
    if (!(depth == 3 || refinement == GTB_REFINEMENT_COARSE)) launch_refine(RM_FIN2, B, T, st, few);
    launch_dp(B, T, DP_TFM_GRAND, 1, 0.0f, 0, 0, 1, st);
    launch_btck(B, T, 1, st);
    launch_alnstr(B, T, st);
    launch_refine(RM_PROD1, B, T, st, few);
    if (refinement == GTB_REFINEMENT_LOG) {
        // MpStageFin.h:421-434: the log search, one launch per step
        Bat TL = T;
        for (int r = 0; r < PLOG_ROUNDS; r++) {
            TL.plog_round = r;
            launch_refine(RM_PLOG, B, TL, st, few);
        }
    } else {
        launch_refine(RM_PROD2, B, T, st, few);
    }
    launch_polish_final(B, T, polish_steps, st);
    launch_final(B, T, referenced, st);
    mark(4);
}

}  // namespace gtb
