// gtb_frg3.cu -- the spatial-index detailed search on sm_100a.
//
// The stage MpStageFrg3::Run (src/libmymp/mpstage1/MpStageFrg3.h:80-115,
// MpStageFrg3.cpp:35-469; GPU form custage1/custage_frg3.cu:54-560) between
// stage 1 and stage 2, for every pair that is not filtered out, each pair as
// if alone in its chunk:
//  1. a local alignment of the two structures by secondary structure, kept
//     as one score byte per cell (k_f3_localdp);
//  2. a grid of configurations (query position x reference position, steps
//     by length and --depth): those whose local score passes the --trigger
//     test are seeded by the local alignment through a cell of the
//     configuration (or by a gapless fragment, --seedrule 0), superposed, and
//     twice re-aligned by each residue's nearest neighbour in the other
//     structure's 3-d tree (first among residues of the same secondary
//     structure) and re-superposed; the final superposition's order-dependent
//     score goes to fragment slot (configuration count mod 32), which keeps
//     its best (k_f3_search, a warp per pair);
//  3. each slot's transform is scored by a gap-0 DP (k_f3_dpscore), the
//     slots ordered by that score, and the best --nbranches refined by DP +
//     fragment refinement (the stage-1 kernels), keeping the best branch;
//  4. two DP refinements start from the best branch.
// Numeric form as elsewhere: FP32 with explicit FMAs, covariance sums over
// position slots in blocks of 32 reduced by xor-shuffle trees and folded into
// Neumaier totals, FP64 rotation solve.  Bit-identical to the oracle's
// frg3_stage.
#include "gtb200.h"
#include "gtb_device.cuh"
#include "gtb_kernels.cuh"

namespace gtb {

namespace {

constexpr int F3_MAXVISIT = 64;     // CUSF_TBSP_INDEX_SCORE_MAXDEPTH
constexpr int F3_HASH = 512;        // CUSF_TBSP_INDEX_SCORE_POSLIMIT2
constexpr int F3_SIMROWS = 96;      // MPSF_TBSP_LOCAL_SIMILARITY_YDIM x 3
constexpr int F3_SIMCOLS = 128;     // MPSF_TBSP_LOCAL_SIMILARITY_XDIM
constexpr int F3_MAXSTACK = 17;
constexpr int F3_LENTHR = 150;      // MpStageFrg3.cpp:48: longer structures thin the sections
constexpr float F3_SSDST2 = 64.f;   // an SS-matched neighbour farther than 8 A is none
constexpr int F3_MAXWIN = 512;      // the largest --window
constexpr int F3_WARPS = 4;         // warps per CTA of the search
constexpr int F3_PERWARP = 4;       // configurations per warp in a round of the search
constexpr int F3_ROUND = F3_WARPS * F3_PERWARP;
// the search's dynamic shared memory: a round's results (scored flags, then
// score + transform per configuration and fragment)
constexpr int F3_ROUND_BYTES = F3_ROUND * 2 * (int)sizeof(int) + F3_ROUND * 2 * 13 * (int)sizeof(float);

__device__ __forceinline__ int pair_q(const Blk& B, const Bat& T, int i) { return (int)((T.p0 + i) / B.nr); }
__device__ __forceinline__ int pair_r(const Blk& B, const Bat& T, int i) { return (int)((T.p0 + i) % B.nr); }

// ---------------------------------------------------------------------------
// 1. Local alignment by secondary structure (ExecDPSSLocal128xKernel,
// MpDPHub.cpp:1256-1480): +1 for equal, -1 for different SS, floored at 0
// (STOP), gap cost per step; the byte per cell is the truncated score
// rounded down to a multiple of 4 (mod 256) with the direction in its low
// two bits.  A warp per pair sweeps strips of 32 rows (a row per lane)
// along anti-diagonals; the previous strip's last row is kept in the pair's
// row buffer.
__global__ void __launch_bounds__(128) k_f3_localdp(Blk B, Bat T) {
    const unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const int slot = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (slot >= T.rhist[RL_NBUCKET]) return;
    const int i = T.rlist[slot];
    const int qi = pair_q(B, T, i), ri = pair_r(B, T, i);
    const int lq = B.qlen[qi], lr = B.rlen[ri];
    const char* qs = B.qs + B.qoff[qi];
    const char* rs = B.rs + B.roff[ri];
    unsigned char* m = T.lsm + T.off_lsm[i];
    float* row = T.row + T.off_row[i];
    const float g = B.f3gapcost;
    const int nstrips = (lq + 31) >> 5;
    for (int s = 0; s < nstrips; s++) {
        const int y = s * 32 + lane;
        const bool valid = y < lq;
        const char qss = valid ? qs[y] : 0;
        float h = 0.f;          // this lane's cell of the previous step: (y, j-1)
        float uplast = 0.f;     // (y-1, j-1)
        unsigned char* my = m + (long long)(valid ? y : 0) * lr;
        for (int t = 0; t < lr + 31; t++) {
            const int j = t - lane;
            float up = __shfl_up_sync(FULL, h, 1);          // lane-1's (y-1, j)
            if (lane == 0) up = (s > 0 && 0 <= j && j < lr) ? row[j] : 0.f;
            if (valid && 0 <= j && j < lr) {
                float dg = j > 0 ? uplast : 0.f;
                float v = __fadd_rn(__fsub_rn((float)((qss == rs[j]) * 2), 1.0f), dg);
                int bk = BT_DIAG;
                if (v < 0.f) { v = 0.f; bk = BT_STOP; }
                const float l = __fadd_rn(j > 0 ? h : 0.f, g);
                if (v < l) { v = l; bk = BT_LEFT; }
                const float u = __fadd_rn(up, g);
                if (v < u) { v = u; bk = BT_UP; }
                h = v;
                my[j] = (unsigned char)((((unsigned)v) & 0xfcu) | (unsigned)bk);
                // lane 31's row is the next strip's "up" (lane 0 of this strip
                // read row[j] 31 steps ago)
                if (lane == 31) row[j] = v;
            }
            uplast = up;
        }
        __syncwarp();           // the row buffer before the next strip reads it
    }
}

// ---------------------------------------------------------------------------
// 2. The configurations of a pair.

// fragment lengths (GetNAlnPoss_frg, covariancebase.h:93-110)
__device__ __forceinline__ int f3_fraglen(int lq, int lr, int fi, int seedrule) {
    const int minlen = lq < lr ? lq : lr;
    const int half = minlen >> 1;
    if (seedrule) return seedrule < half ? seedrule : half;
    if (fi == 0) {
        int leno3 = (int)__fmul_rn((float)minlen, 1.0f / 3.0f);
        if (leno3 < 1) leno3 = 1;
        return leno3 < 20 ? leno3 : 20;
    }
    return half < 100 ? half : 100;
}

// configuration position step (GetFragStepSize_frg_*, covariancebase.h:22-84)
__device__ __forceinline__ int f3_step(int depth, int len) {
    int leno3 = (int)__fmul_rn((float)len, 1.0f / 3.0f);
    if (leno3 < 1) leno3 = 1;
    const int small = leno3 < 15 ? leno3 : 15;
    if (depth == 0) return len > 150 ? 15 : small;
    if (depth == 1) return len > 150 ? 23 : small;
    const int med = len > 250 ? 45 : len > 200 ? 35 : len > 150 ? 25 : small;
    return depth == 2 ? med : 2 * med;
}

__device__ __forceinline__ float warp_max(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// the xor-shuffle tree sum of a warp (every lane gets it)
__device__ __forceinline__ float tree32(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = __fadd_rn(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// The local similarity test (CalcLocalSimilarity2_frg2,
// MpStageFrg3.h:327-415): the largest score byte over 96 rows from qrypos
// and up to 128 columns from rfnpos (rounded up to a multiple of 4) reaches
// the fragment length x the trigger fraction.
__device__ bool f3_similar(const unsigned char* m, int lq, int lr, int qrypos, int rfnpos, int fl,
                           float thr, int lane) {
    if (lq < qrypos + fl) fl = lq - qrypos;
    if (lr < rfnpos + fl) fl = lr - rfnpos;
    int pidelta = (lr - 3 - rfnpos) & ~3;
    if (pidelta > F3_SIMCOLS) pidelta = F3_SIMCOLS;
    const int pibeg = (rfnpos + 3) & ~3;
    unsigned mx = 0;
    for (int ii = 0; qrypos + ii < lq && ii < F3_SIMROWS; ii++) {
        const unsigned char* rowp = m + (long long)(qrypos + ii) * lr + pibeg;
        for (int c = lane; c < pidelta; c += 32) {
            const unsigned v = rowp[c] & 0xfcu;
            mx = v > mx ? v : mx;
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const unsigned w = __shfl_xor_sync(0xffffffffu, mx, o);
        mx = w > mx ? w : mx;
    }
    return !(__fmul_rn((float)fl, thr) > (float)mx);
}

// Seed from the local alignment (CalcCCMatricesLocallyAligned_Complete,
// MpStage1.h:395-470), on lane 0: of 4 evenly spaced cells the first with
// the largest byte, the local alignment traced back from it inside the
// rectangle from (qrypos, rfnpos); the pairs go to pq/pr in increasing order.
// Returns their number (0: too few), the same on every lane.
__device__ int f3_seed_local(const unsigned char* m, int lq, int lr, int trig, int fraglen,
                             int qrypos, int rfnpos, int* pq, int* pr, int lane) {
    int n = 0;
    if (lane == 0) {
        if (lq < qrypos + fraglen && lr < rfnpos + fraglen)
            fraglen = (lq - qrypos) > (lr - rfnpos) ? (lq - qrypos) : (lr - rfnpos);
        fraglen >>= 2;
        int y = qrypos, x = rfnpos;
        float vr = 0.f;
        for (int f = 0; f < 4; f++) {
            int yt = qrypos + (f + 1) * fraglen, xt = rfnpos + (f + 1) * fraglen;
            yt = yt < lq - 1 ? yt : lq - 1;
            xt = xt < lr - 1 ? xt : lr - 1;
            const float vrt = (float)(m[(long long)yt * lr + xt] & 0xfcu);
            if (vr < vrt) { vr = vrt; y = yt; x = xt; }
        }
        while (y >= qrypos && x >= rfnpos && n < F3_MAXWIN) {
            const int b = m[(long long)y * lr + x] & 3;
            if (b == BT_STOP) break;
            if (b == BT_UP) { y--; continue; }
            if (b == BT_LEFT) { x--; continue; }
            pq[n] = y; pr[n] = x; n++;
            x--; y--;
        }
        const int minf = fraglen < 16 ? fraglen : 16;
        if (n < 1 || (trig && n < minf)) n = 0;
        for (int a = 0, b = n - 1; a < b; a++, b--) {
            int t = pq[a]; pq[a] = pq[b]; pq[b] = t;
            t = pr[a]; pr[a] = pr[b]; pr[b] = t;
        }
    }
    __syncwarp();
    return __shfl_sync(0xffffffffu, n, 0);
}

// Covariance sums over position slots 0..n-1 (pq/pr; a negative index: no
// pair): lane k of block b takes slot 32b + k; each block's values are
// summed by the xor-shuffle tree and folded into Neumaier totals in block
// order.  Every lane gets the 16 values (15 sums and the count).
__device__ void f3_cov(const float* qx, const float* qy, const float* qz, const float* rx,
                       const float* ry, const float* rz, const int* pq, const int* pr, int n,
                       float* v, int lane) {
    float s[15], c[15];
#pragma unroll
    for (int f = 0; f < 15; f++) { s[f] = 0.f; c[f] = 0.f; }
    int cnt = 0;
    for (int b0 = 0; b0 < n; b0 += 32) {
        const int k = b0 + lane;
        const int a = k < n ? pq[k] : -1, b = k < n ? pr[k] : -1;
        const bool ok = a >= 0 && b >= 0;
        const float x0 = ok ? qx[a] : 0.f, y0 = ok ? qy[a] : 0.f, z0 = ok ? qz[a] : 0.f;
        const float x1 = ok ? rx[b] : 0.f, y1 = ok ? ry[b] : 0.f, z1 = ok ? rz[b] : 0.f;
        float t[15] = {__fmul_rn(x0, x1), __fmul_rn(x0, y1), __fmul_rn(x0, z1),
                       __fmul_rn(y0, x1), __fmul_rn(y0, y1), __fmul_rn(y0, z1),
                       __fmul_rn(z0, x1), __fmul_rn(z0, y1), __fmul_rn(z0, z1),
                       x0, y0, z0, x1, y1, z1};
#pragma unroll
        for (int f = 0; f < 15; f++) {
            float bs = tree32(t[f]);
            nfold(s[f], c[f], bs);
        }
        cnt += __popc(__ballot_sync(0xffffffffu, ok));
    }
#pragma unroll
    for (int f = 0; f < 15; f++) v[f] = __fadd_rn(s[f], c[f]);
    v[15] = (float)cnt;
}

// Nearest neighbour in a structure's 3-d tree (NNByIndex*,
// MpStageFrg3.h:1270-1440): depth first with a bounded stack, at most 64
// nodes visited; with ssfilt only residues of secondary structure ss count
// and one farther than 8 A is none.  Returns the residue or -1.  Nodes are
// packed (k_pack_nodes): nd = (x, y, z, residue | SS << 16), nc = (left,
// right).  The stack is the lane's column of a shared-memory array (entry q
// at [q * 32]).
__device__ int f3_nn(const float4* nd, const int2* nc, int len, bool ssfilt, char ss, float px,
                     float py, float pz, int stacksize, unsigned short* stk_node, float* stk_diff,
                     unsigned char* stk_dim) {
    int sp = 0, nvisited = 0, best = -1, root = len >> 1, dim = 0;
    float bestd = 9.9e6f;
    while (0 < sp || 0 <= root) {
        if (0 <= root) {
            nvisited++;
            if (F3_MAXVISIT <= nvisited) break;
            const float4 n = __ldg(nd + root);
            const int2 ch = __ldg(nc + root);
            const int ow = __float_as_int(n.w);
            const int org = ow & 0xffff;
            const float dx = __fsub_rn(n.x, px), dy = __fsub_rn(n.y, py), dz = __fsub_rn(n.z, pz);
            const float d2 = __fmaf_rn(dx, dx, __fmaf_rn(dy, dy, __fmul_rn(dz, dz)));
            if ((best < 0 || d2 < bestd) && (!ssfilt || (char)(ow >> 16) == ss)) {
                bestd = d2;
                best = org;
            }
            if (bestd == 0.0f) break;
            const float diffc = dim == 0 ? dx : (dim == 1 ? dy : dz);
            if (2 < ++dim) dim = 0;
            if (sp < stacksize) {
                stk_node[sp * 32] = (unsigned short)root;    // a node index is below 65536
                stk_dim[sp * 32] = (unsigned char)dim;
                stk_diff[sp * 32] = diffc;
                sp++;
            }
            root = (0.0f < diffc) ? ch.x : ch.y;
        } else {
            bool cond = false;
            float diffc = 0.f;
            while (0 < sp && !cond) {
                sp--;
                root = stk_node[sp * 32]; dim = stk_dim[sp * 32]; diffc = stk_diff[sp * 32];
                cond = __fmul_rn(diffc, diffc) < bestd;
            }
            if (!cond) break;
            const int2 ch = __ldg(nc + root);
            root = (0.0f < diffc) ? ch.y : ch.x;
        }
    }
    if (ssfilt) return F3_SSDST2 < bestd ? -1 : best;
    return best;
}

// per-pair view of the search's inputs
struct F3Pair {
    int lq, lr;
    const float *qx, *qy, *qz, *rx, *ry, *rz;
    const char *qs, *rs;
    const float4 *qnd, *rnd;
    const int2 *qnc, *rnc;
};

// Neighbours over the window of the shorter structure
// (ProduceAlignmentUsingIndex2Reference/Query, MpStageFrg3.h:500-680), a
// window slot per lane per round; fills pq/pr (-1: empty), returns the
// window length.
__device__ int f3_window(const F3Pair& P, const float* tfm, bool ssfilt, int window, int qrypos,
                         int rfnpos, int stacksize, int* pq, int* pr, int lane, unsigned short* sn,
                         float* sd, unsigned char* sm) {
    const int lq = P.lq, lr = P.lr;
    int n;
    if (lq < lr) {
        const int fl = lr < window ? lr : window;
        int qp = qrypos - (fl >> 1); if (qp < 0) qp = 0;
        const int ql = qp + fl < lq ? qp + fl : lq;
        qp = ql - fl; if (qp < 0) qp = 0;
        n = ql - qp;
        for (int pi = lane; pi < n; pi += 32) {
            const int q = qp + pi;
            float x, y, z;
            xform(tfm, P.qx[q], P.qy[q], P.qz[q], x, y, z);
            const int r = f3_nn(P.rnd, P.rnc, lr, ssfilt, P.qs[q], x, y, z, stacksize, sn, sd, sm);
            pq[pi] = q;
            pr[pi] = r > 0 ? r : -1;
        }
    } else {
        const int fl = lq < window ? lq : window;
        int rp = rfnpos - (fl >> 1); if (rp < 0) rp = 0;
        const int rl = rp + fl < lr ? rp + fl : lr;
        rp = rl - fl; if (rp < 0) rp = 0;
        n = rl - rp;
        for (int pi = lane; pi < n; pi += 32) {
            const int r = rp + pi;
            float x, y, z;
            xform(tfm, P.rx[r], P.ry[r], P.rz[r], x, y, z);
            const int q = f3_nn(P.qnd, P.qnc, lq, ssfilt, P.rs[r], x, y, z, stacksize, sn, sd, sm);
            pq[pi] = q > 0 ? q : -1;
            pr[pi] = r;
        }
    }
    __syncwarp();
    return n;
}

// The order-dependent score (CalcScoresUnrl_SWFTscanProgressive_Complete,
// MpStageFrg3.h:760-850) over the first cnt window slots: each pair extends
// the best chain of earlier-partnered pairs kept in a 512-entry table hashed
// by partner index; lanes share the table scan, lane 0 updates it.
//
// When the partner structure has at most F3_HASH residues no two partners
// share an entry, so an entry only ever rises (to the larger chain score of
// its own partner) and the scan "best entry with a lower partner" is the
// running maximum of the entries below the partner's: the table is then
// kept as prefix maxima (pm[k] = max of entries 0..k), read with one load
// and raised by every lane for its own entries at or above the partner's.
__device__ float f3_progressive(const F3Pair& P, const float* tfm, float d02, const int* pq,
                                const int* pr, int cnt, bool partner_is_r, float* omax,
                                float* ondx, int lane) {
    if ((partner_is_r ? P.lr : P.lq) <= F3_HASH) {
        float* pm = omax;
        for (int k = lane; k < F3_HASH; k += 32) pm[k] = 0.f;
        __syncwarp();
        for (int pi = 0; pi < cnt; pi++) {
            const int a = pq[pi], b = pr[pi];
            if (a < 0 || b < 0) continue;          // the same on every lane
            const float d = dist2_tf(tfm, P.qx[a], P.qy[a], P.qz[a], P.rx[b], P.ry[b], P.rz[b]);
            const float sco = tmterm(d02, d);
            if (!(0.f < sco)) continue;
            const int c = partner_is_r ? b : a;
            const float mx = c > 0 ? pm[c - 1] : 0.f;
            const float nsc = __fadd_rn(mx, sco);
            __syncwarp();
            for (int k = c + ((lane - c) & 31); k < F3_HASH; k += 32) pm[k] = fmaxf(pm[k], nsc);
            __syncwarp();
        }
        const float mx = pm[F3_HASH - 1];
        __syncwarp();
        return mx;
    }
    for (int k = lane; k < F3_HASH; k += 32) { omax[k] = 0.f; ondx[k] = -1.f; }
    __syncwarp();
    for (int pi = 0; pi < cnt; pi++) {
        const int a = pq[pi], b = pr[pi];
        if (a < 0 || b < 0) continue;          // the same on every lane
        const float d = dist2_tf(tfm, P.qx[a], P.qy[a], P.qz[a], P.rx[b], P.ry[b], P.rz[b]);
        const float sco = tmterm(d02, d);
        if (!(0.f < sco)) continue;
        const float qnx = (float)(partner_is_r ? b : a);
        float mx = 0.f;
        for (int k = lane; k < F3_HASH; k += 32)
            if (ondx[k] < qnx && mx < omax[k]) mx = omax[k];
        mx = warp_max(mx);
        if (lane == 0) {
            const int c = (int)qnx & (F3_HASH - 1);
            const float st = ondx[c], ss = omax[c], nsc = __fadd_rn(mx, sco);
            const bool half2nd = pi > (cnt >> 1);
            if (st < 0.f || (st == qnx && ss < nsc) || ((half2nd && st < qnx) || (!half2nd && qnx < st))) {
                ondx[c] = qnx;
                omax[c] = nsc;
            }
        }
        __syncwarp();
    }
    float mx = 0.f;
    for (int k = lane; k < F3_HASH; k += 32) mx = mx < omax[k] ? omax[k] : mx;
    mx = warp_max(mx);
    __syncwarp();
    return mx;
}

__device__ __forceinline__ int f3_stacksize(int lq, int lr) {
    const int L = lq > lr ? lq : lr;
    int b = L > 1 ? 32 - __clz(L - 1) : 0;    // ceil(log2 L)
    b += 1;
    return b < F3_MAXSTACK ? b : F3_MAXSTACK;
}

// A CTA per listed pair; a round is F3_ROUND consecutive configurations,
// F3_PERWARP per warp (interleaved, so that cheap and dear ones mix); a
// scored configuration's slot is the pair's count of scored configurations
// before it mod 32, and the slot keeps its best: after each round the
// round's results are applied in configuration order, as one warp going
// through the configurations in order would.
__global__ void __launch_bounds__(F3_WARPS * 32, 3) k_f3_search(Blk B, Bat T, int depth) {
    __shared__ int s_pq[F3_WARPS][F3_MAXWIN], s_pr[F3_WARPS][F3_MAXWIN];
    __shared__ float s_omax[F3_WARPS][F3_HASH], s_ondx[F3_WARPS][F3_HASH];
    __shared__ unsigned short s_stkn[F3_WARPS][F3_MAXSTACK * 32];
    __shared__ float s_stkd[F3_WARPS][F3_MAXSTACK * 32];
    __shared__ unsigned char s_stkm[F3_WARPS][F3_MAXSTACK * 32];
    // a round's results (F3_ROUND_BYTES, dynamic): per configuration of the
    // round and fragment, scored (1) or not; score and transform
    extern __shared__ float s_dyn[];
    int* s_got = (int*)s_dyn;
    float* s_res = s_dyn + F3_ROUND * 2;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int slot = blockIdx.x;
    if (slot >= T.rhist[RL_NBUCKET]) return;       // the same for the whole CTA
    const int i = T.rlist[slot];
    const int qi = pair_q(B, T, i), ri = pair_r(B, T, i);
    F3Pair P;
    P.lq = B.qlen[qi]; P.lr = B.rlen[ri];
    const int qo = B.qoff[qi], ro = B.roff[ri];
    P.qx = B.qx + qo; P.qy = B.qy + qo; P.qz = B.qz + qo;
    P.rx = B.rx + ro; P.ry = B.ry + ro; P.rz = B.rz + ro;
    P.qs = B.qs + qo; P.rs = B.rs + ro;
    P.qnd = B.qnd + qo; P.qnc = B.qnc + qo;
    P.rnd = B.rnd + ro; P.rnc = B.rnc + ro;
    const int lq = P.lq, lr = P.lr;
    const int ml = lq < lr ? lq : lr;
    const float d0 = B.t_d0[ml];
    const float d02 = __fmul_rn(d0, d0);
    const unsigned char* m = T.lsm + T.off_lsm[i];
    int* pq = s_pq[w];
    int* pr = s_pr[w];
    unsigned short* sn = s_stkn[w] + lane;
    float* sd = s_stkd[w] + lane;
    unsigned char* sm = s_stkm[w] + lane;
    const int nsec = B.f3nsec;
    float* slots = T.f3slot + (long long)i * nsec * F3_NTOP * 13;
    for (int k = threadIdx.x; k < nsec * F3_NTOP; k += blockDim.x) slots[k * 13] = 0.f;
    const float thr = __fdiv_rn((float)B.f3trigger, 100.0f);
    const int seedrule = B.f3seedrule;
    const int qstep = f3_step(depth, lq), rstep = f3_step(depth, lr);
    const int minn = depth == 3 ? 5 : 10;
    int nsy = lq / qstep + 1; if (nsy < minn) nsy = minn;
    int nsx = lr / rstep + 1; if (nsx < minn) nsx = minn;
    const int nconf = nsy * nsx;
    const int stacksize = f3_stacksize(lq, lr);
    const int f0 = f3_fraglen(lq, lr, 0, 0), f1 = f3_fraglen(lq, lr, 1, 0);
    const int nfr = seedrule ? 1 : 2;
    int nscored = 0;                              // kept by thread 0
    for (int c0 = 0; c0 < nconf; c0 += F3_ROUND)
    for (int jj = 0; jj <= F3_PERWARP; jj++) {
      if (jj == F3_PERWARP) {
        // the round's results in configuration order
        __syncthreads();
        if (threadIdx.x == 0) {
            for (int rr = 0; rr < F3_ROUND; rr++) {
                // the sections this configuration feeds: section 0 all; at
                // --depth 1 and 0 sections 1 and 2 those on every second /
                // third grid row and column of a structure longer than
                // F3_LENTHR (sec2met, sec3met: MpStageFrg3.cpp:204-212)
                const int cc = c0 + rr, ys = cc / nsx, xs = cc % nsx;
                const bool sec1 = nsec > 1 && (lq <= F3_LENTHR || (ys & 1) == 0) &&
                                  (lr <= F3_LENTHR || (xs & 1) == 0);
                const bool sec2 = nsec > 2 && (lq <= F3_LENTHR || ys % 3 == 0) &&
                                  (lr <= F3_LENTHR || xs % 3 == 0);
                for (int fi = 0; fi < 2; fi++) {
                    if (!s_got[rr * 2 + fi]) continue;
                    const int k = nscored % F3_NTOP;
                    nscored++;
                    const float* res = s_res + (rr * 2 + fi) * 13;
                    const float sc = res[0];
                    if (!(0.0f < sc)) continue;
                    for (int sec = 0; sec < nsec; sec++) {
                        if ((sec == 1 && !sec1) || (sec == 2 && !sec2)) continue;
                        float* sl = slots + (sec * F3_NTOP + k) * 13;
                        if (sl[0] < sc) {
                            sl[0] = sc;
                            for (int f = 0; f < 12; f++) sl[1 + f] = res[1 + f];
                        }
                    }
                }
            }
        }
        __syncthreads();
        continue;
      }
        const int rix = w + F3_WARPS * jj;        // this configuration's place in the round
        const int c = c0 + rix;
        if (lane < 2) s_got[rix * 2 + lane] = 0;
        __syncwarp();
        if (c < nconf) {
            const int qrypos = (c / nsx) * qstep, rfnpos = (c % nsx) * rstep;
            bool go = !(lq < qrypos + f0 || lr < rfnpos + f0 || f0 < 1);
            const bool conv1 = (lq < qrypos + f1 || lr < rfnpos + f1 || f1 < 1);
            if (go && 0.0f < thr && !f3_similar(m, lq, lr, qrypos, rfnpos, f1, thr, lane)) go = false;
            for (int fi = 0; go && fi < nfr; fi++) {
                if (fi == 1 && conv1) continue;
                const int fraglen = fi == 0 ? f0 : f1;
                if (lq < qrypos + fraglen || lr < rfnpos + fraglen) continue;
                float v[16], tfm[12];
                int n;
                if (seedrule) {
                    n = f3_seed_local(m, lq, lr, B.f3trigger > 0, f3_fraglen(lq, lr, fi, seedrule),
                                      qrypos, rfnpos, pq, pr, lane);
                } else {
                    for (int k = lane; k < fraglen; k += 32) { pq[k] = qrypos + k; pr[k] = rfnpos + k; }
                    __syncwarp();
                    n = fraglen;
                }
                if (n < 1) continue;
                f3_cov(P.qx, P.qy, P.qz, P.rx, P.ry, P.rz, pq, pr, n, v, lane);
                __syncwarp();
                if (v[15] < 1.0f) continue;
                solve_sums(v, lq < lr ? 0 : 2, tfm);
                for (int it = 0; it < 2; it++) {
                    const int cw = f3_window(P, tfm, it == 0, B.f3window, qrypos, rfnpos, stacksize,
                                             pq, pr, lane, sn, sd, sm);
                    f3_cov(P.qx, P.qy, P.qz, P.rx, P.ry, P.rz, pq, pr, cw, v, lane);
                    if (v[15] < 1.0f) { __syncwarp(); continue; }
                    if (it == 0) { solve_sums(v, lq < lr ? 0 : 2, tfm); __syncwarp(); continue; }
                    solve_sums(v, 0, tfm);
                    const float sc = f3_progressive(P, tfm, d02, pq, pr, (int)v[15], lq < lr,
                                                    s_omax[w], s_ondx[w], lane);
                    if (lane == 0) {
                        float* res = s_res + (rix * 2 + fi) * 13;
                        s_got[rix * 2 + fi] = 1;
                        res[0] = sc;
#pragma unroll
                        for (int f = 0; f < 12; f++) res[1 + f] = tfm[f];
                    }
                    __syncwarp();
                }
            }
        }
    }
}

// ---------------------------------------------------------------------------
// 3. Per section, the slots by DP score (SortBestDPscoresAndTMsAmongDPswifts,
// MpStageFrg3.h:1150-1250), larger first, lower slot first on ties: the
// pair's flag becomes section 0's first slot's (SCOREDP when no slot scored),
// the first --nbranches of each section are its branches (branch index =
// section * nbranches + rank), and the next DP refinement skips refinement
// variant section * 32 + rank when that rank holds no score (section 0's
// rank 0 being the pair's flag).  A thread per pair.
__global__ void k_f3_select(Blk B, Bat T, int nbranches) {
    const int slot = blockIdx.x * blockDim.x + threadIdx.x;
    if (slot >= T.rhist[RL_NBUCKET]) return;
    const int i = T.rlist[slot];
    const int nsec = B.f3nsec;
    for (int sec = 0; sec < F3_NSEC; sec++) {
        if (sec >= nsec) { T.vskip_mask[(long long)i * F3_NSEC + sec] = 0u; continue; }
        const float* dps = T.f3dps + ((long long)i * nsec + sec) * F3_NTOP;
        float d[F3_NTOP];
        int order[F3_NTOP];
        for (int k = 0; k < F3_NTOP; k++) { d[k] = dps[k]; order[k] = k; }
        for (int a = 1; a < F3_NTOP; a++) {
            const int k = order[a];
            int b = a - 1;
            while (b >= 0 && d[order[b]] < d[k]) { order[b + 1] = order[b]; b--; }
            order[b + 1] = k;
        }
        unsigned vs = 0u;
        for (int r = sec == 0 ? 1 : 0; r < F3_NTOP; r++)
            if (!(0.0f < d[order[r]])) vs |= 1u << r;
        T.vskip_mask[(long long)i * F3_NSEC + sec] = vs;
        if (sec == 0) T.flags[i] = 0.0f < d[order[0]] ? 0 : CONV_SCOREDP;
        for (int r = 0; r < nbranches; r++) {
            const int k = order[r];
            const bool ok = 0.0f < d[k];
            const long long br = (long long)i * T.f3br + sec * nbranches + r;
            T.f3ok[br] = ok ? 1 : 0;
            if (ok) {
                const float* src = T.f3slot + (((long long)i * nsec + sec) * F3_NTOP + k) * 13 + 1;
                float* dst = T.f3alt + br * 12;
                for (int f = 0; f < 12; f++) dst[f] = src[f];
            }
        }
    }
}

// The best branch so far (SaveBestScoreAndTMAmongBests with a secondary
// update, MpStageBase.h:1250-1310): after branch rci, its refinement result
// (score and iteration-best transform) replaces the kept one for the first
// branch, or when it scores higher.  A thread per listed pair.
__global__ void k_f3_second(Blk B, Bat T, int rci) {
    const int slot = blockIdx.x * blockDim.x + threadIdx.x;
    if (slot >= T.rhist[RL_NBUCKET]) return;
    const int i = T.rlist[slot];
    const float b = T.best[i];
    if (rci == 0 || T.best2[i] < b) {
        T.best2[i] = b;
        for (int f = 0; f < 12; f++) T.tfm_2nd[i * 12 + f] = T.tfm_ib[i * 12 + f];
    }
}

}  // namespace

// The stage over a batch (the pairs not filtered out).  The pair list is
// built once; the stage-1 kernels (DP, traceback, refinement) build their
// own lists, so the frg3 list is rebuilt before each frg3 kernel that
// reads it.
void launch_frg3(const Blk& B, const Bat& T, cudaStream_t st) {
    const int nb = (T.np + 3) / 4;
    auto plist = [&]() { launch_pair_list(B, T, CONV_LOWTMSC, st); };
    plist();
    const int nbr = B.f3nbranches < F3_NBMAX ? B.f3nbranches : F3_NBMAX;
    {
        KtScope kts(T, KF_FRG3, st);
        if (0 < B.f3trigger || B.f3seedrule) {
            k_f3_localdp<<<nb, 128, 0, st>>>(B, T);
            if (T.launches) (*T.launches)++;
        }
        // static arrays (~48 kB) + the round's results go past the default 48 kB
        cudaFuncSetAttribute(k_f3_search, cudaFuncAttributeMaxDynamicSharedMemorySize, F3_ROUND_BYTES);
        k_f3_search<<<T.np, F3_WARPS * 32, F3_ROUND_BYTES, st>>>(B, T, B.depth);
        if (T.launches) (*T.launches)++;
        launch_f3_dpscore(B, T, st);
        k_f3_select<<<(T.np + 255) / 256, 256, 0, st>>>(B, T, nbr);
        if (T.launches) (*T.launches)++;
    }
    // the branches, section by section (Refine_tfmaltconfig,
    // MpStageFrg3.cpp:425-467); at --depth 1 and 0 each branch's refinement
    // is followed by a DP under its iteration-best transform and a
    // refinement of that alignment (MpStageFrg3.cpp:452-466)
    for (int rci = 0; rci < B.f3nsec * nbr; rci++) {
        Bat TA = T;
        TA.alt_rci = rci;
        launch_dp(B, TA, DP_TFM_ALT, 1, 0.0f, 0, 0, 0, st);
        launch_btck(B, TA, 0, st);
        launch_refine(RM_DP, B, T, st, true);
        plist();
        k_f3_second<<<(T.np + 255) / 256, 256, 0, st>>>(B, T, rci);
        if (T.launches) (*T.launches)++;
        if (B.depth <= 1) {
            launch_dp(B, T, DP_TFM_IBEST, 1, 0.0f, 0, 0, 0, st);
            launch_btck(B, T, 0, st);
            launch_refine(RM_DP, B, T, st, true);
            plist();
            k_f3_second<<<(T.np + 255) / 256, 256, 0, st>>>(B, T, rci);
            if (T.launches) (*T.launches)++;
        }
    }
    // DP refinement from the best branch, with a gap cost (its refinements
    // skipping the variants the slots rule out) and without
    // (MpStageFrg3.h:108-112)
    Bat TV = T;
    TV.vskip = T.vskip_mask;
    launch_dprefine(B, TV, 0, 0, 2, 0.0f, true, DP_TFM_2ND, st);
    launch_dprefine(B, T, 1, 0, 2, 0.0f, true, DP_TFM_IBEST, st);
}

}  // namespace gtb
