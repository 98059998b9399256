// gtb_adjoint.cu -- TM-score adjoint for fixed alignments and projected-
// gradient polishing of superpositions on SO(3) x R^3.
//
// For a pair with aligned residues (q_i, r_i), transform (R, t) and d0:
//   e_i = R q_i + t - r_i,  u_i = d0^2 + |e_i|^2,  TM = sum_i d0^2 / u_i
//   dTM/de_i = -2 d0^2 e_i / u_i^2
//   dTM/dt      = sum_i dTM/de_i
//   dTM/domega  = sum_i (R q_i) x dTM/de_i     (R <- exp([omega]x) R)
//   dTM/dq_i    = R^T dTM/de_i
// One warp per pair; lanes stride over residues; FP32 arithmetic with
// per-lane compensated sums and a fixed butterfly reduction.
#include <cuda_runtime.h>
#include <cstdio>
#include "gtb200.h"
#include "gtb_device.cuh"
#include "gtb_kernels.cuh"

namespace {

__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

struct Kahan {
    float s = 0.f, c = 0.f;
    __device__ __forceinline__ void add(float x) {
        float y = x - c;
        float t = s + y;
        c = (t - s) - y;
        s = t;
    }
    // c holds the rounding excess of the last additions: the compensated
    // total is s - c
    __device__ __forceinline__ float value() const { return s - c; }
};

// TM-score and gradient for one pair; omega about the point `cen`
// (cen = 0 gives the public origin-based derivative).
template <int S>
__device__ void tm_grad(const float* q, const float* r, int n, const float* T, float d0,
                        const float* cen, float* gq, float& tm, float* g6) {
    int lane = threadIdx.x & 31;
    float d02 = d0 * d0;
    Kahan s, gw[3], gt[3];
    for (int i = lane; i < n; i += 32) {
        float qx = q[S * i], qy = q[S * i + 1], qz = q[S * i + 2];
        float px = T[0] * qx + T[1] * qy + T[2] * qz;
        float py = T[3] * qx + T[4] * qy + T[5] * qz;
        float pz = T[6] * qx + T[7] * qy + T[8] * qz;
        float ex = px + T[9] - r[S * i], ey = py + T[10] - r[S * i + 1], ez = pz + T[11] - r[S * i + 2];
        float u = d02 + ex * ex + ey * ey + ez * ez;
        float iu = 1.f / u;
        s.add(d02 * iu);
        float k = -2.f * d02 * iu * iu;
        float gx = k * ex, gy = k * ey, gz = k * ez;
        gt[0].add(gx); gt[1].add(gy); gt[2].add(gz);
        float ax = px + T[9] - cen[0], ay = py + T[10] - cen[1], az = pz + T[11] - cen[2];
        if (cen[0] == 0.f && cen[1] == 0.f && cen[2] == 0.f) { ax = px; ay = py; az = pz; }
        gw[0].add(ay * gz - az * gy);
        gw[1].add(az * gx - ax * gz);
        gw[2].add(ax * gy - ay * gx);
        if (gq) {
            gq[3 * i] = T[0] * gx + T[3] * gy + T[6] * gz;
            gq[3 * i + 1] = T[1] * gx + T[4] * gy + T[7] * gz;
            gq[3 * i + 2] = T[2] * gx + T[5] * gy + T[8] * gz;
        }
    }
    tm = warp_sum(s.value());
    for (int k = 0; k < 3; k++) {
        g6[k] = warp_sum(gw[k].value());
        g6[3 + k] = warp_sum(gt[k].value());
    }
}

__global__ void k_tm_adjoint(int npairs, const long long* off, const int* n, const float* qxyz,
                             const float* rxyz, const float* tfm, const float* d0, float* tm,
                             float* grad, float* gq) {
    int p = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (p >= npairs) return;
    int lane = threadIdx.x & 31;
    long long o = off[p];
    const float zero[3] = {0.f, 0.f, 0.f};
    float T[12];
    for (int f = 0; f < 12; f++) T[f] = tfm[p * 12 + f];
    float t, g6[6];
    tm_grad<3>(qxyz + 3 * o, rxyz + 3 * o, n[p], T, d0[p], zero, gq ? gq + 3 * o : nullptr, t, g6);
    if (lane == 0) {
        if (tm) tm[p] = t;
        if (grad) for (int k = 0; k < 6; k++) grad[p * 6 + k] = g6[k];
    }
}

template <int S>
__device__ float tm_only(const float* q, const float* r, int n, const float* T, float d0) {
    int lane = threadIdx.x & 31;
    float d02 = d0 * d0;
    Kahan s;
    for (int i = lane; i < n; i += 32) {
        float qx = q[S * i], qy = q[S * i + 1], qz = q[S * i + 2];
        float ex = T[0] * qx + T[1] * qy + T[2] * qz + T[9] - r[S * i];
        float ey = T[3] * qx + T[4] * qy + T[5] * qz + T[10] - r[S * i + 1];
        float ez = T[6] * qx + T[7] * qy + T[8] * qz + T[11] - r[S * i + 2];
        s.add(d02 / (d02 + ex * ex + ey * ey + ez * ez));
    }
    return warp_sum(s.value());
}

// curvature scales for the step: h_t = sum 2 d0^2/u^2, h_w = sum 2 d0^2 |a|^2/u^2
template <int S>
__device__ void curvature(const float* q, const float* r, int n, const float* T, float d0,
                          const float* cen, float& ht, float& hw) {
    int lane = threadIdx.x & 31;
    float d02 = d0 * d0;
    float a1 = 0.f, a2 = 0.f;
    for (int i = lane; i < n; i += 32) {
        float qx = q[S * i], qy = q[S * i + 1], qz = q[S * i + 2];
        float px = T[0] * qx + T[1] * qy + T[2] * qz + T[9];
        float py = T[3] * qx + T[4] * qy + T[5] * qz + T[10];
        float pz = T[6] * qx + T[7] * qy + T[8] * qz + T[11];
        float ex = px - r[S * i], ey = py - r[S * i + 1], ez = pz - r[S * i + 2];
        float u = d02 + ex * ex + ey * ey + ez * ez;
        float w = 2.f * d02 / (u * u);
        a1 += w;
        float ax = px - cen[0], ay = py - cen[1], az = pz - cen[2];
        a2 += w * (ax * ax + ay * ay + az * az);
    }
    ht = warp_sum(a1);
    hw = warp_sum(a2);
}

// apply x -> exp([w]x)(x - c) + c + dt to the transform (Rodrigues, FP64)
__device__ void apply_step(const float* T, const float* w, const float* dt, const float* c,
                           float* Tn) {
    double th = sqrt((double)w[0] * w[0] + (double)w[1] * w[1] + (double)w[2] * w[2]);
    double K[9] = {0, -w[2], w[1], w[2], 0, -w[0], -w[1], w[0], 0};
    double A = th > 1e-12 ? sin(th) / th : 1.0;
    double Bc = th > 1e-6 ? (1.0 - cos(th)) / (th * th) : 0.5;
    double K2[9];
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) {
            double s = 0;
            for (int k = 0; k < 3; k++) s += K[3 * i + k] * K[3 * k + j];
            K2[3 * i + j] = s;
        }
    double E[9];
    for (int k = 0; k < 9; k++) E[k] = ((k % 4) == 0 ? 1.0 : 0.0) + A * K[k] + Bc * K2[k];
    double Rn[9];
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) {
            double s = 0;
            for (int k = 0; k < 3; k++) s += E[3 * i + k] * (double)T[3 * k + j];
            Rn[3 * i + j] = s;
        }
    for (int i = 0; i < 3; i++) {
        double s = 0;
        for (int k = 0; k < 3; k++) s += E[3 * i + k] * ((double)T[9 + k] - c[k]);
        Tn[9 + i] = (float)(s + c[i] + dt[i]);
    }
    for (int k = 0; k < 9; k++) Tn[k] = (float)Rn[k];
}

// Projected-gradient ascent of TM (d0) over (R, t) for one pair, from T;
// a step is kept only if it raises the score.  Returns the final score.
template <int S>
__device__ float polish_pair(const float* q, const float* r, int m, float d0, float* T, int steps,
                             float* before) {
    float Tn[12];
    float cur = tm_only<S>(q, r, m, T, d0);
    if (before) *before = cur;
    int lane = threadIdx.x & 31;
    for (int it = 0; it < steps && m > 0; it++) {
        // centroid of the transformed query
        float cx = 0.f, cy = 0.f, cz = 0.f;
        for (int i = lane; i < m; i += 32) {
            float qx = q[S * i], qy = q[S * i + 1], qz = q[S * i + 2];
            cx += T[0] * qx + T[1] * qy + T[2] * qz + T[9];
            cy += T[3] * qx + T[4] * qy + T[5] * qz + T[10];
            cz += T[6] * qx + T[7] * qy + T[8] * qz + T[11];
        }
        float c[3] = {warp_sum(cx) / m, warp_sum(cy) / m, warp_sum(cz) / m};
        float tmv, g6[6], ht, hw;
        tm_grad<S>(q, r, m, T, d0, c, nullptr, tmv, g6);
        curvature<S>(q, r, m, T, d0, c, ht, hw);
        if (!(ht > 0.f) || !(hw > 0.f)) break;
        float w[3] = {g6[0] / hw, g6[1] / hw, g6[2] / hw};
        float dt[3] = {g6[3] / ht, g6[4] / ht, g6[5] / ht};
        bool acc = false;
        for (int bt = 0; bt < 10 && !acc; bt++) {
            apply_step(T, w, dt, c, Tn);
            float nv = tm_only<S>(q, r, m, Tn, d0);
            if (nv > cur) {
                acc = true;
                cur = nv;
                for (int f = 0; f < 12; f++) T[f] = Tn[f];
            } else {
                for (int k = 0; k < 3; k++) { w[k] *= 0.5f; dt[k] *= 0.5f; }
            }
        }
        if (!acc) break;
    }
    return cur;
}

__global__ void k_polish(int npairs, const long long* off, const int* n, const float* qxyz,
                         const float* rxyz, float* tfm, const float* d0v, int steps,
                         float* tmb, float* tma) {
    int p = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (p >= npairs) return;
    int lane = threadIdx.x & 31;
    long long o = off[p];
    float T[12], before;
    for (int f = 0; f < 12; f++) T[f] = tfm[p * 12 + f];
    float cur = polish_pair<3>(qxyz + 3 * o, rxyz + 3 * o, n[p], d0v[p], T, steps, &before);
    if (lane == 0) {
        for (int f = 0; f < 12; f++) tfm[p * 12 + f] = T[f];
        if (tmb) tmb[p] = before;
        if (tma) tma[p] = cur;
    }
}

// Polishing inside the search, after the production scores: each pair's
// final transform is polished against TM with the search's d0 (that of the
// shorter structure) over its final alignment (the aligned coordinates the
// traceback stored, 6 floats per aligned pair); when a step was kept, the
// FP32 TM-scores by both lengths are recomputed for the new transform (the
// FP64 recomputation and error record follow in the final kernel).
__global__ void k_polish_final(gtb::Blk B, gtb::Bat T, int steps) {
    int i = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (i >= T.np) return;
    int lane = threadIdx.x & 31;
    if (T.flags[i] & gtb::CONV_LOWTMSC) return;
    int m = T.naln[i];
    if (m < 3) return;
    int qi = (int)((T.p0 + i) / B.nr), ri = (int)((T.p0 + i) % B.nr);
    int lq = B.qlen[qi], lr = B.rlen[ri];
    int ml = lq < lr ? lq : lr;
    const float* q = T.alc + 6 * T.off_aln[i];
    const float* r = q + 3;
    float Tm[12], before;
    for (int f = 0; f < 12; f++) Tm[f] = T.tfm_gr[i * 12 + f];
    float cur = polish_pair<6>(q, r, m, B.t_d0fin[ml], Tm, steps, &before);
    if (!(cur > before)) return;
    float tq = tm_only<6>(q, r, m, Tm, B.t_d0fin[lq]);
    float tr = tm_only<6>(q, r, m, Tm, B.t_d0fin[lr]);
    if (lane == 0) {
        for (int f = 0; f < 12; f++) T.tfm_gr[i * 12 + f] = Tm[f];
        T.out[i * 16 + 9] = tq / (float)lq;
        T.out[i * 16 + 10] = tr / (float)lr;
    }
}

}  // namespace

namespace gtb {
void launch_polish_final(const Blk& B, const Bat& T, int steps, cudaStream_t st) {
    if (steps <= 0 || T.np <= 0) return;
    k_polish_final<<<(T.np + 3) / 4, 128, 0, st>>>(B, T, steps);
    if (T.launches) (*T.launches)++;
}
}  // namespace gtb

struct gtb_handle;
extern "C" gtb_status gtb_tm_adjoint(gtb_handle* h, int npairs, const long long* off, const int* n,
                                     const float* qxyz, const float* rxyz, const float* tfm,
                                     const float* d0, float* tm, float* grad, float* gq, void* stream) {
    (void)h;
    if (npairs < 0 || !off || !n || !qxyz || !rxyz || !tfm || !d0) return GTB_ERR_ARG;
    if (npairs == 0) return GTB_OK;
    int blocks = (npairs + 3) / 4;
    k_tm_adjoint<<<blocks, 128, 0, (cudaStream_t)stream>>>(npairs, off, n, qxyz, rxyz, tfm, d0, tm, grad, gq);
    return cudaGetLastError() == cudaSuccess ? GTB_OK : GTB_ERR_CUDA;
}

extern "C" gtb_status gtb_polish(gtb_handle* h, int npairs, const long long* off, const int* n,
                                 const float* qxyz, const float* rxyz, float* tfm, const float* d0,
                                 int steps, float* tm_before, float* tm_after, void* stream) {
    (void)h;
    if (npairs < 0 || !off || !n || !qxyz || !rxyz || !tfm || !d0 || steps < 0) return GTB_ERR_ARG;
    if (npairs == 0) return GTB_OK;
    int blocks = (npairs + 3) / 4;
    k_polish<<<blocks, 128, 0, (cudaStream_t)stream>>>(npairs, off, n, qxyz, rxyz, tfm, d0, steps,
                                                       tm_before, tm_after);
    return cudaGetLastError() == cudaSuccess ? GTB_OK : GTB_ERR_CUDA;
}
