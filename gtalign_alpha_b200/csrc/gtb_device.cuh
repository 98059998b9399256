// gtb_device.cuh -- device primitives of the superposition search.
//
// Arithmetic is written out explicitly so that the device results are a
// fixed function of the inputs: every fused multiply-add is an explicit
// __fmaf_rn and the translation unit is compiled with -fmad=false, divisions
// and square roots are the IEEE-rounded forms.  The same operations in the
// same order give the same floats on any IEEE-754 machine.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace gtb {

constexpr int   BLK = 32;                 // positions per compensated block
constexpr float LARGEDST = 999999.9f;     // stagecnsts.cuh:15
constexpr float LARGEDST_CMP = 399999.9f; // stagecnsts.cuh:17
constexpr float RM_CONVEPS = 1.e-5f;      // stagecnsts.cuh:42
constexpr float SCORE_CONVEPS = 1.e-6f;   // scoringbase.h:36
constexpr int   FRAG_NSUB = 6;            // mpprocconfbase.h:28
constexpr int   FRAG_STEP = 40;           // mpprocconfbase.h:30
constexpr int   NMAXCONVIT = 20;          // mpprocconfbase.h:33
constexpr int   FIN_MAXNPOS = 128;        // mpprocconfbase.h:73
constexpr int   MINFRAGLEN = 4;           // GetMinFragLengthForAln for lengths >= 96
constexpr int   CONV_SCOREDP = 2;         // gproc.h:40
constexpr int   CONV_LOWTMSC = 8;         // gproc.h:46
enum { BT_STOP = 0, BT_LEFT = 1, BT_UP = 2, BT_DIAG = 3 };  // gproc.h:176-181

// ---------------------------------------------------------------------------
__device__ __forceinline__ void xform(const float* t, float x, float y, float z,
                                      float& ox, float& oy, float& oz) {
    ox = __fmaf_rn(t[0], x, __fmaf_rn(t[1], y, __fmaf_rn(t[2], z, t[9])));
    oy = __fmaf_rn(t[3], x, __fmaf_rn(t[4], y, __fmaf_rn(t[5], z, t[10])));
    oz = __fmaf_rn(t[6], x, __fmaf_rn(t[7], y, __fmaf_rn(t[8], z, t[11])));
}
__device__ __forceinline__ float dist2(float ax, float ay, float az,
                                       float bx, float by, float bz) {
    float dx = __fsub_rn(ax, bx), dy = __fsub_rn(ay, by), dz = __fsub_rn(az, bz);
    return __fmaf_rn(dx, dx, __fmaf_rn(dy, dy, __fmul_rn(dz, dz)));
}
__device__ __forceinline__ float dist2_tf(const float* t, float qx, float qy, float qz,
                                          float rx, float ry, float rz) {
    float x, y, z;
    xform(t, qx, qy, qz, x, y, z);
    return dist2(x, y, z, rx, ry, rz);
}
__device__ __forceinline__ float tmterm(float d02, float d) {
    return __fdiv_rn(d02, __fadd_rn(d02, d));
}

// Neumaier fold of a block partial b into the compensated total (s, c).
__device__ __forceinline__ void nfold(float& s, float& c, float& b) {
    float t = __fadd_rn(s, b);
    if (fabsf(s) >= fabsf(b)) c = __fadd_rn(c, __fadd_rn(__fsub_rn(s, t), b));
    else c = __fadd_rn(c, __fadd_rn(__fsub_rn(b, t), s));
    s = t;
    b = 0.f;
}

// Compensated covariance accumulator: 9 cross products, 2x3 coordinate sums.
struct CovAcc {
    float s[15], c[15], b[15];
    int n;
    __device__ __forceinline__ void init() {
#pragma unroll
        for (int f = 0; f < 15; f++) { s[f] = 0.f; c[f] = 0.f; b[f] = 0.f; }
        n = 0;
    }
    __device__ __forceinline__ void add(float qx, float qy, float qz,
                                        float rx, float ry, float rz) {
        b[0] = __fmaf_rn(qx, rx, b[0]); b[1] = __fmaf_rn(qx, ry, b[1]); b[2] = __fmaf_rn(qx, rz, b[2]);
        b[3] = __fmaf_rn(qy, rx, b[3]); b[4] = __fmaf_rn(qy, ry, b[4]); b[5] = __fmaf_rn(qy, rz, b[5]);
        b[6] = __fmaf_rn(qz, rx, b[6]); b[7] = __fmaf_rn(qz, ry, b[7]); b[8] = __fmaf_rn(qz, rz, b[8]);
        b[9] = __fadd_rn(b[9], qx); b[10] = __fadd_rn(b[10], qy); b[11] = __fadd_rn(b[11], qz);
        b[12] = __fadd_rn(b[12], rx); b[13] = __fadd_rn(b[13], ry); b[14] = __fadd_rn(b[14], rz);
        n++;
    }
    __device__ __forceinline__ void fold() {
#pragma unroll
        for (int f = 0; f < 15; f++) nfold(s[f], c[f], b[f]);
    }
    // 16 values: 15 sums + n
    __device__ __forceinline__ void final(float* v) {
        fold();
#pragma unroll
        for (int f = 0; f < 15; f++) v[f] = __fadd_rn(s[f], c[f]);
        v[15] = (float)n;
    }
};

// ---------------------------------------------------------------------------
// FP64 rotation solve: Horn's quaternion key matrix, largest eigenvalue by
// Newton iteration on its characteristic quartic (Theobald 2005, QCP), the
// eigenvector from the adjugate of (N - lambda I).
__device__ __forceinline__ double det3(double a, double b, double c, double d, double e,
                                       double f, double g, double h, double i) {
    return __dadd_rn(__dsub_rn(__dmul_rn(a, __dsub_rn(__dmul_rn(e, i), __dmul_rn(f, h))),
                               __dmul_rn(b, __dsub_rn(__dmul_rn(d, i), __dmul_rn(f, g)))),
                     __dmul_rn(c, __dsub_rn(__dmul_rn(d, h), __dmul_rn(e, g))));
}

__device__ __forceinline__ double cof4(const double (&M)[4][4], int i, int j) {
    double m[9];
    int k = 0;
#pragma unroll
    for (int r = 0; r < 4; r++) {
        if (r == i) continue;
#pragma unroll
        for (int c = 0; c < 4; c++) {
            if (c == j) continue;
            m[k++] = M[r][c];
        }
    }
    double d = det3(m[0], m[1], m[2], m[3], m[4], m[5], m[6], m[7], m[8]);
    return ((i + j) & 1) ? -d : d;
}

__device__ __forceinline__ double qcp_lambda(const double (&S)[3][3], double (&N)[4][4]) {
    double Sxx = S[0][0], Sxy = S[0][1], Sxz = S[0][2];
    double Syx = S[1][0], Syy = S[1][1], Syz = S[1][2];
    double Szx = S[2][0], Szy = S[2][1], Szz = S[2][2];
    N[0][0] = __dadd_rn(__dadd_rn(Sxx, Syy), Szz);
    N[0][1] = __dsub_rn(Syz, Szy); N[0][2] = __dsub_rn(Szx, Sxz); N[0][3] = __dsub_rn(Sxy, Syx);
    N[1][1] = __dsub_rn(__dsub_rn(Sxx, Syy), Szz);
    N[1][2] = __dadd_rn(Sxy, Syx); N[1][3] = __dadd_rn(Szx, Sxz);
    N[2][2] = __dsub_rn(__dadd_rn(-Sxx, Syy), Szz);
    N[2][3] = __dadd_rn(Syz, Szy);
    N[3][3] = __dadd_rn(__dsub_rn(-Sxx, Syy), Szz);
    N[1][0] = N[0][1]; N[2][0] = N[0][2]; N[3][0] = N[0][3];
    N[2][1] = N[1][2]; N[3][1] = N[1][3]; N[3][2] = N[2][3];
    double ss = 0.0;
#pragma unroll
    for (int a = 0; a < 3; a++)
#pragma unroll
        for (int b = 0; b < 3; b++) ss = __dadd_rn(ss, __dmul_rn(S[a][b], S[a][b]));
    double c2 = __dmul_rn(-2.0, ss);
    double c1 = __dmul_rn(-8.0, det3(Sxx, Sxy, Sxz, Syx, Syy, Syz, Szx, Szy, Szz));
    double c0 = 0.0;
#pragma unroll
    for (int j = 0; j < 4; j++) c0 = __dadd_rn(c0, __dmul_rn(N[0][j], cof4(N, 0, j)));
    double lam = __dsqrt_rn(__dmul_rn(3.0, ss));
    double lam0 = lam;
    for (int it = 0; it < 50; it++) {
        double l2 = __dmul_rn(lam, lam);
        double p = __dadd_rn(__dadd_rn(__dmul_rn(__dadd_rn(l2, c2), l2), __dmul_rn(c1, lam)), c0);
        double dp = __dadd_rn(__dadd_rn(__dmul_rn(__dmul_rn(4.0, l2), lam),
                                        __dmul_rn(__dmul_rn(2.0, c2), lam)), c1);
        if (!(dp != 0.0)) break;
        double step = __ddiv_rn(p, dp);
        lam = __dsub_rn(lam, step);
        if (fabs(step) <= __dmul_rn(1.e-13, lam0)) break;
    }
    return lam;
}

__device__ __forceinline__ int qcp_rotation(const double (&S)[3][3], double (&R)[9]) {
    double N[4][4];
    double lam = qcp_lambda(S, N);
#pragma unroll
    for (int i = 0; i < 4; i++) N[i][i] = __dsub_rn(N[i][i], lam);
    double dg[4];
    int jm = 0;
#pragma unroll
    for (int j = 0; j < 4; j++) {
        dg[j] = cof4(N, j, j);
        if (fabs(dg[j]) > fabs(dg[jm])) jm = j;
    }
    double dgm = dg[0];
    if (jm == 1) dgm = dg[1];
    if (jm == 2) dgm = dg[2];
    if (jm == 3) dgm = dg[3];
    double l3 = __dmul_rn(__dmul_rn(fabs(lam), lam), lam);
    if (!(fabs(dgm) > __dmul_rn(1.e-14, l3)) || !(lam > 0.0)) return 0;
    double q[4], qn = 0.0;
#pragma unroll
    for (int i = 0; i < 4; i++) { q[i] = cof4(N, i, jm); qn = __dadd_rn(qn, __dmul_rn(q[i], q[i])); }
    if (!(qn > 0.0)) return 0;
    qn = __ddiv_rn(1.0, __dsqrt_rn(qn));
    double a = __dmul_rn(q[0], qn), b = __dmul_rn(q[1], qn), c = __dmul_rn(q[2], qn), d = __dmul_rn(q[3], qn);
    double aa = __dmul_rn(a, a), bb = __dmul_rn(b, b), cc = __dmul_rn(c, c), dd = __dmul_rn(d, d);
    R[0] = __dsub_rn(__dsub_rn(__dadd_rn(aa, bb), cc), dd);
    R[1] = __dmul_rn(2.0, __dsub_rn(__dmul_rn(b, c), __dmul_rn(a, d)));
    R[2] = __dmul_rn(2.0, __dadd_rn(__dmul_rn(b, d), __dmul_rn(a, c)));
    R[3] = __dmul_rn(2.0, __dadd_rn(__dmul_rn(b, c), __dmul_rn(a, d)));
    R[4] = __dsub_rn(__dadd_rn(__dsub_rn(aa, bb), cc), dd);
    R[5] = __dmul_rn(2.0, __dsub_rn(__dmul_rn(c, d), __dmul_rn(a, b)));
    R[6] = __dmul_rn(2.0, __dsub_rn(__dmul_rn(b, d), __dmul_rn(a, c)));
    R[7] = __dmul_rn(2.0, __dadd_rn(__dmul_rn(c, d), __dmul_rn(a, b)));
    R[8] = __dadd_rn(__dsub_rn(__dsub_rn(aa, bb), cc), dd);
    return 1;
}

// sums v: [0..8] sum q_i r_j, [9..11] sum q, [12..14] sum r, [15] n.
// swap 1: solve with the reference rotated onto the query, then invert
// (--symmetric for a shorter query, MpStageBase.h:1000-1023); swap 2: the
// reference rotated onto the query, not inverted (the detailed search's
// orientation towards the longer structure, MpStageBase.h:1086-1101).
static __device__ __noinline__ void solve_sums(const float* v, int swap, float* tfm) {
    double dn = (double)v[15];
    double mq[3], mr[3], S[3][3];
#pragma unroll
    for (int i = 0; i < 3; i++) {
        mq[i] = __ddiv_rn((double)v[9 + i], dn);
        mr[i] = __ddiv_rn((double)v[12 + i], dn);
    }
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) {
            double x = swap ? (double)v[3 * j + i] : (double)v[3 * i + j];
            double m = swap ? __dmul_rn(__dmul_rn(dn, mq[j]), mr[i]) : __dmul_rn(__dmul_rn(dn, mq[i]), mr[j]);
            S[i][j] = __dsub_rn(x, m);
        }
    double R[9];
    int ok = qcp_rotation(S, R);
    if (!ok) {
#pragma unroll
        for (int k = 0; k < 9; k++) R[k] = 0.0;
        R[0] = R[4] = R[8] = 1.0;
    }
    if (!swap) {
#pragma unroll
        for (int i = 0; i < 3; i++) {
            double t = __dsub_rn(mr[i], __dadd_rn(__dadd_rn(__dmul_rn(R[3 * i], mq[0]),
                                                           __dmul_rn(R[3 * i + 1], mq[1])),
                                                 __dmul_rn(R[3 * i + 2], mq[2])));
            tfm[9 + i] = (float)t;
        }
#pragma unroll
        for (int k = 0; k < 9; k++) tfm[k] = (float)R[k];
    } else if (swap == 2) {
#pragma unroll
        for (int i = 0; i < 3; i++)
            tfm[9 + i] = (float)__dsub_rn(mq[i], __dadd_rn(__dadd_rn(__dmul_rn(R[3 * i], mr[0]),
                                                                     __dmul_rn(R[3 * i + 1], mr[1])),
                                                           __dmul_rn(R[3 * i + 2], mr[2])));
#pragma unroll
        for (int k = 0; k < 9; k++) tfm[k] = (float)R[k];
    } else {
        double t[3];
#pragma unroll
        for (int i = 0; i < 3; i++)
            t[i] = __dsub_rn(mq[i], __dadd_rn(__dadd_rn(__dmul_rn(R[3 * i], mr[0]),
                                                       __dmul_rn(R[3 * i + 1], mr[1])),
                                             __dmul_rn(R[3 * i + 2], mr[2])));
#pragma unroll
        for (int i = 0; i < 3; i++)
#pragma unroll
            for (int j = 0; j < 3; j++) tfm[3 * i + j] = (float)R[3 * j + i];
#pragma unroll
        for (int i = 0; i < 3; i++)
            tfm[9 + i] = (float)(-__dadd_rn(__dadd_rn(__dmul_rn(R[i], t[0]), __dmul_rn(R[3 + i], t[1])),
                                            __dmul_rn(R[6 + i], t[2])));
    }
}

// RMSD of the optimal superposition from FP64 sums (21 values: 15 as above,
// then sum q^2 (3), sum r^2 (3)), n pairs.
__device__ __forceinline__ double rmsd_from_sums(const double* v, double n) {
    double mq[3], mr[3], S[3][3], E0 = 0.0;
#pragma unroll
    for (int i = 0; i < 3; i++) { mq[i] = __ddiv_rn(v[9 + i], n); mr[i] = __ddiv_rn(v[12 + i], n); }
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) S[i][j] = __dsub_rn(v[3 * i + j], __dmul_rn(__dmul_rn(n, mq[i]), mr[j]));
#pragma unroll
    for (int i = 0; i < 3; i++)
        E0 = __dadd_rn(E0, __dadd_rn(__dsub_rn(v[15 + i], __dmul_rn(__dmul_rn(n, mq[i]), mq[i])),
                                     __dsub_rn(v[18 + i], __dmul_rn(__dmul_rn(n, mr[i]), mr[i]))));
    double N[4][4];
    double lam = qcp_lambda(S, N);
    double e = __ddiv_rn(__dsub_rn(E0, __dmul_rn(2.0, lam)), n);
    return e > 0.0 ? __dsqrt_rn(e) : 0.0;
}

// fragment rules: fragment.cuh:30-110
__device__ __forceinline__ int frag_length(int alnlen, int sfragndx) {
    if (alnlen < 4 && sfragndx == 0) return alnlen;
    int a = alnlen >> sfragndx;
    if (a == 2 && 0 < sfragndx && ((alnlen >> (sfragndx - 1)) & 1)) a = 4;
    if (a < 3) return 0;
    if (a < 4) a = 4;
    if (sfragndx + 1 == FRAG_NSUB) a = 4;
    return a;
}
__device__ __forceinline__ float d0s_of(float d0) {
    float d = d0 < 8.f ? d0 : 8.f;
    return d > 4.5f ? d : 4.5f;
}

}  // namespace gtb
