/*
 * gtoracle.c -- CPU oracle (checker) for the GTalign superposition search.
 *
 * TEST INFRASTRUCTURE ONLY: loaded by tests/, __graft_entry__.smoke() and
 * bench.py's cpu_baseline leg; never by the product.
 *
 * A sequential restatement, one query-reference pair at a time, of the
 * reference's CPU stage sequence:
 *   MpBatch::ProcessBlock           src/libmymp/mpbatch/MpBatch.cpp:208-470
 *   MpStageFrg3::Run (the spatial-index detailed search, each pair as if alone
 *     in its chunk on one thread)   src/libmymp/mpstage1/MpStageFrg3.h:80-115,
 *                                   MpStageFrg3.cpp:35-469,
 *     ExecDPSSLocal128xKernel       src/libmymp/mpdp/MpDPHub.cpp:1256-1480,
 *     ExecDPScore128xKernel         src/libmymp/mpdp/MpDPHub.cpp:389-645
 *   MpStage1::Preinitialize1Kernel  src/libmymp/mpstage1/MpStage1.cpp:28-167
 *   MpSecStr::ssk_kernel_helper     src/libmymp/mpss/MpSecStr.cpp:26-118,
 *                                   AassignSecStr src/libmymp/mpss/MpSecStr.h:218-249
 *   MpStage1::FindFragKernel        src/libmymp/mpstage1/MpStage1.cpp:289-440
 *   MpStage1::RefineFragInitKernel  src/libmymp/mpstage1/MpStage1.cpp:548-736
 *   MpStage1::DPRefine              src/libmymp/mpstage1/MpStage1.cpp:466-517
 *   MpStage1::RefineFragDPKernel    src/libmymp/mpstage1/MpStage1.cpp:760-948
 *   MpStage2::RunSpecialized/Align  src/libmymp/mpstage1/MpStage2.h:63-126
 *   MpStageFin::Run                 src/libmymp/mpstage1/MpStageFin.h:63-96
 *   MpDPHub::ExecDPwBtck128xKernel  src/libmymp/mpdp/MpDPHub.cpp:72-346 and
 *     ExecDPTFMSSwBtck128xKernel    src/libmymp/mpdp/MpDPHub.cpp:686-940
 *   MpDPHub::BtckToMatched128x      src/libmymp/mpdp/MpDPHub.cpp:1515-1660
 *   MpDPHub::ConstrainedBtck...     src/libmymp/mpdp/MpDPHub.cpp:1699-1905
 *   MpDPHub::ProductionMatchTo...   src/libmymp/mpdp/MpDPHub.cpp:1919-2125
 *   MpStageFin production kernels   src/libmymp/mpstage1/MpStageFin.cpp:747-1525
 *   constants (d0, d8, d0s)         src/libmycu/custages/stagecnsts.cuh:48-175
 *   fragment rules                  src/libmycu/custages/fragment.cuh:30-110
 *
 * Numeric form (shared with the CUDA path so the two agree bit for bit):
 *  - FP32 coordinates; transforms and squared distances written with explicit
 *    fmaf at fixed places; nothing else contracted (-ffp-contract=off);
 *  - every sum over positions is accumulated in forward position order in
 *    FP32 blocks of GTB_BLK positions (the absolute blocks [32m, 32m+32) of
 *    the position space), each block folded into a Neumaier compensated
 *    FP32 total;
 *  - rotation solve in FP64 by the quaternion characteristic polynomial
 *    (Horn 1987; Theobald 2005 "QCP"): Newton iteration for the largest
 *    eigenvalue, eigenvector from the adjugate of (K - lambda I);
 *  - the reported TM-scores and RMSD are recomputed in FP64 from the final
 *    alignment and transform; |FP32 path - FP64| is reported per pair.
 *  - d0 / d8 constants are FP32 values of the reference formulas
 *    (cbrtf/powf of glibc), tabulated per length on the host.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include "gtoracle.h"
#include "../gtalign_alpha_b200/csrc/gtb_gonnet.h"

#define GTB_BLK 32
#define LARGEDST 999999.9f
#define LARGEDST_CMP 399999.9f
#define RM_CONVEPS 1.e-5f
#define SCORE_CONVEPS 1.e-6f
#define FRAG_NSUB 6
/* stored --refinement codes, command line code + 1 (CLOptions.h:121-128) */
#define REF_LOG 0
#define REF_COARSE 1
#define REF_ONE 2
#define REF_FULL 3
#define REF_FULLA 4
#define FRAG_STEP 40
#define NMAXCONVIT 20
#define FIN_MAXNPOS 128
#define MINFRAGLEN 4

#define CONV_SCOREDP 2
#define CONV_LOWTMSC 8

enum { BT_STOP = 0, BT_LEFT = 1, BT_UP = 2, BT_DIAG = 3 };

/* ------------------------------------------------------------------------ */
/* constants: stagecnsts.cuh:48-175                                          */
static float c_d0(int lq, int lr) {
    float l = (float)(lq < lr ? lq : lr);
    float d0 = 0.168f;
    if (l > 19.f) d0 = 1.24f * cbrtf(l - 15.f) - 1.8f;
    return d0 + 0.8f;
}
static float c_d82(int lq, int lr) {
    float l = (float)(lq < lr ? lq : lr);
    float d8 = 1.5f * powf(l, 0.3f) + 3.5f;
    return d8 * d8;
}
static float c_d0fin(int lq, int lr) {
    float l = (float)(lq < lr ? lq : lr);
    float d0 = 0.5f;
    if (l > 21.f) d0 = 1.24f * cbrtf(l - 15.f) - 1.8f;
    if (d0 < 0.5f) d0 = 0.5f;
    return d0;
}
/* GetD0finNA, stagecnsts.cuh:93-106: the final d0 of a nucleic-acid pair */
static float c_d0fin_na(int lq, int lr) {
    float l = (float)(lq < lr ? lq : lr);
    float d0 = 0.3f;
    if (30.f <= l) d0 = 0.6f * sqrtf(l - 0.5f) - 2.5f;
    else if (23.f < l) d0 = 0.7f;
    else if (19.f < l) d0 = 0.6f;
    else if (15.f < l) d0 = 0.5f;
    else if (11.f < l) d0 = 0.4f;
    return d0 > 0.3f ? d0 : 0.3f;
}
/* GetD0fin(l1, l2, type), stagecnsts.cuh:108-114: type of the reference structure */
static float c_d0fin_t(int lq, int lr, int na) { return na ? c_d0fin_na(lq, lr) : c_d0fin(lq, lr); }
static float c_d0s(float d0) {
    float d = d0;
    d = d < 8.f ? d : 8.f;
    d = d > 4.5f ? d : 4.5f;
    return d;
}
void gto_constants(int lq, int lr, float* d0, float* d02, float* d82,
                   float* d0fin, float* d02dpscan) {
    float a = c_d0(lq, lr);
    if (d0) *d0 = a;
    if (d02) *d02 = a * a;
    if (d82) *d82 = c_d82(lq, lr);
    if (d0fin) *d0fin = c_d0fin(lq, lr);
    if (d02dpscan) { float b = a + 1.5f; *d02dpscan = b * b; }
}

/* fragment.cuh:30-110 */
static int frag_length(int alnlen, int sfragndx) {
    if (alnlen < 4 && sfragndx == 0) return alnlen;
    int a = alnlen >> sfragndx;
    if (a == 2 && 0 < sfragndx && ((alnlen >> (sfragndx - 1)) & 1)) a = 4;
    if (a < 3) return 0;
    if (a < 4) a = 4;
    if (sfragndx + 1 == FRAG_NSUB) a = 4;
    return a;
}
static int max_nfrag_steps(int maxalnlen, int step, int fraglen) {
    return (int)ceilf((float)(maxalnlen + step - fraglen) / step);
}

/* ------------------------------------------------------------------------ */
/* geometry primitives (fixed FMA placement)                                 */
static inline void xform(const float* t, float x, float y, float z,
                         float* ox, float* oy, float* oz) {
    *ox = fmaf(t[0], x, fmaf(t[1], y, fmaf(t[2], z, t[9])));
    *oy = fmaf(t[3], x, fmaf(t[4], y, fmaf(t[5], z, t[10])));
    *oz = fmaf(t[6], x, fmaf(t[7], y, fmaf(t[8], z, t[11])));
}
static inline float dist2_tf(const float* t, float qx, float qy, float qz,
                             float rx, float ry, float rz) {
    float x, y, z;
    xform(t, qx, qy, qz, &x, &y, &z);
    float dx = x - rx, dy = y - ry, dz = z - rz;
    return fmaf(dx, dx, fmaf(dy, dy, dz * dz));
}

/* ------------------------------------------------------------------------ */
/* block-compensated sums                                                    */
static inline void nfold(float* s, float* c, float* b) {
    float t = *s + *b;
    if (fabsf(*s) >= fabsf(*b)) *c += (*s - t) + *b;
    else *c += (*b - t) + *s;
    *s = t;
    *b = 0.f;
}

typedef struct { float s[15], c[15], b[15]; int n; } ccacc;
static void cc_init(ccacc* a) { memset(a, 0, sizeof(*a)); }
static inline void cc_add(ccacc* a, float qx, float qy, float qz,
                          float rx, float ry, float rz) {
    a->b[0] = fmaf(qx, rx, a->b[0]); a->b[1] = fmaf(qx, ry, a->b[1]); a->b[2] = fmaf(qx, rz, a->b[2]);
    a->b[3] = fmaf(qy, rx, a->b[3]); a->b[4] = fmaf(qy, ry, a->b[4]); a->b[5] = fmaf(qy, rz, a->b[5]);
    a->b[6] = fmaf(qz, rx, a->b[6]); a->b[7] = fmaf(qz, ry, a->b[7]); a->b[8] = fmaf(qz, rz, a->b[8]);
    a->b[9] += qx; a->b[10] += qy; a->b[11] += qz;
    a->b[12] += rx; a->b[13] += ry; a->b[14] += rz;
    a->n++;
}
static inline void cc_fold(ccacc* a) { for (int f = 0; f < 15; f++) nfold(&a->s[f], &a->c[f], &a->b[f]); }
/* final: 16 values (15 sums + n) */
static void cc_final(ccacc* a, float* v) {
    cc_fold(a);
    for (int f = 0; f < 15; f++) v[f] = a->s[f] + a->c[f];
    v[15] = (float)a->n;
}

/* ------------------------------------------------------------------------ */
/* FP64 rotation solve (quaternion characteristic polynomial)               */
static double det3(double a, double b, double c, double d, double e, double f,
                   double g, double h, double i) {
    return a * (e * i - f * h) - b * (d * i - f * g) + c * (d * h - e * g);
}
/* cofactor (i,j) of symmetric 4x4 M */
static double cof4(const double M[4][4], int i, int j) {
    double m[9];
    int k = 0;
    for (int r = 0; r < 4; r++) {
        if (r == i) continue;
        for (int c = 0; c < 4; c++) {
            if (c == j) continue;
            m[k++] = M[r][c];
        }
    }
    double d = det3(m[0], m[1], m[2], m[3], m[4], m[5], m[6], m[7], m[8]);
    return ((i + j) & 1) ? -d : d;
}

/* Largest eigenvalue of Horn's key matrix for S (S[a][b] = sum x_a y_b,
 * centred).  Returns lambda; fills N. */
static double qcp_lambda(const double S[3][3], double N[4][4]) {
    double Sxx = S[0][0], Sxy = S[0][1], Sxz = S[0][2];
    double Syx = S[1][0], Syy = S[1][1], Syz = S[1][2];
    double Szx = S[2][0], Szy = S[2][1], Szz = S[2][2];
    N[0][0] = Sxx + Syy + Szz; N[0][1] = Syz - Szy; N[0][2] = Szx - Sxz; N[0][3] = Sxy - Syx;
    N[1][1] = Sxx - Syy - Szz; N[1][2] = Sxy + Syx; N[1][3] = Szx + Sxz;
    N[2][2] = -Sxx + Syy - Szz; N[2][3] = Syz + Szy;
    N[3][3] = -Sxx - Syy + Szz;
    N[1][0] = N[0][1]; N[2][0] = N[0][2]; N[3][0] = N[0][3];
    N[2][1] = N[1][2]; N[3][1] = N[1][3]; N[3][2] = N[2][3];
    double ss = 0.0;
    for (int a = 0; a < 3; a++)
        for (int b = 0; b < 3; b++) ss += S[a][b] * S[a][b];
    double c2 = -2.0 * ss;
    double c1 = -8.0 * det3(Sxx, Sxy, Sxz, Syx, Syy, Syz, Szx, Szy, Szz);
    /* det(N) by cofactor expansion along row 0 */
    double c0 = 0.0;
    for (int j = 0; j < 4; j++) c0 += N[0][j] * cof4(N, 0, j);
    double lam = sqrt(3.0 * ss);
    double lam0 = lam;
    for (int it = 0; it < 50; it++) {
        double l2 = lam * lam;
        double p = (l2 + c2) * l2 + c1 * lam + c0;
        double dp = 4.0 * l2 * lam + 2.0 * c2 * lam + c1;
        if (!(dp != 0.0)) break;
        double step = p / dp;
        lam -= step;
        if (fabs(step) <= 1.e-13 * lam0) break;
    }
    return lam;
}

/* Rotation (row-major) rotating x onto y from S; returns 0 on degenerate. */
static int qcp_rotation(const double S[3][3], double R[9], double* lamout) {
    double N[4][4];
    double lam = qcp_lambda(S, N);
    if (lamout) *lamout = lam;
    for (int i = 0; i < 4; i++) N[i][i] -= lam;
    double dg[4];
    int jm = 0;
    for (int j = 0; j < 4; j++) {
        dg[j] = cof4(N, j, j);
        if (fabs(dg[j]) > fabs(dg[jm])) jm = j;
    }
    double l3 = fabs(lam) * lam * lam;
    if (!(fabs(dg[jm]) > 1.e-14 * l3) || !(lam > 0.0)) return 0;
    double q[4], qn = 0.0;
    for (int i = 0; i < 4; i++) { q[i] = cof4(N, i, jm); qn += q[i] * q[i]; }
    if (!(qn > 0.0)) return 0;
    qn = 1.0 / sqrt(qn);
    double a = q[0] * qn, b = q[1] * qn, c = q[2] * qn, d = q[3] * qn;
    R[0] = a * a + b * b - c * c - d * d; R[1] = 2.0 * (b * c - a * d);     R[2] = 2.0 * (b * d + a * c);
    R[3] = 2.0 * (b * c + a * d);     R[4] = a * a - b * b + c * c - d * d; R[5] = 2.0 * (c * d - a * b);
    R[6] = 2.0 * (b * d - a * c);     R[7] = 2.0 * (c * d + a * b);     R[8] = a * a - b * b - c * c + d * d;
    return 1;
}

/* sums: [0..8] sum q_i r_j, [9..11] sum q, [12..14] sum r; n.
 * swap 0: tfm rotates/translates the query onto the reference (row-major R,
 * t); 1: solved with the reference moving onto the query, then inverted
 * (--symmetric); 2: the reference moving onto the query, not inverted (the
 * detailed search's orientation towards the longer structure,
 * MpStageBase.h:1086-1101). */
static int solve_sums(const float* v, int n, int swap, float* tfm) {
    double dn = (double)n;
    double mq[3], mr[3], S[3][3];
    for (int i = 0; i < 3; i++) { mq[i] = (double)v[9 + i] / dn; mr[i] = (double)v[12 + i] / dn; }
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++)
            S[i][j] = (double)v[3 * i + j] - dn * mq[i] * mr[j];
    double R[9];
    int ok;
    if (!swap) {
        ok = qcp_rotation(S, R, NULL);
        if (!ok) { memset(R, 0, sizeof(R)); R[0] = R[4] = R[8] = 1.0; }
        double t[3];
        for (int i = 0; i < 3; i++) t[i] = mr[i] - (R[3*i] * mq[0] + R[3*i+1] * mq[1] + R[3*i+2] * mq[2]);
        for (int k = 0; k < 9; k++) tfm[k] = (float)R[k];
        for (int i = 0; i < 3; i++) tfm[9 + i] = (float)t[i];
    } else {
        /* rotate the reference onto the query, then invert */
        double St[3][3];
        for (int i = 0; i < 3; i++)
            for (int j = 0; j < 3; j++) St[i][j] = S[j][i];
        ok = qcp_rotation(St, R, NULL);
        if (!ok) { memset(R, 0, sizeof(R)); R[0] = R[4] = R[8] = 1.0; }
        double t[3];
        for (int i = 0; i < 3; i++) t[i] = mq[i] - (R[3*i] * mr[0] + R[3*i+1] * mr[1] + R[3*i+2] * mr[2]);
        if (swap == 2) {
            for (int k = 0; k < 9; k++) tfm[k] = (float)R[k];
            for (int i = 0; i < 3; i++) tfm[9 + i] = (float)t[i];
            return ok;
        }
        /* inverse: R^T, -R^T t */
        for (int i = 0; i < 3; i++)
            for (int j = 0; j < 3; j++) tfm[3 * i + j] = (float)R[3 * j + i];
        for (int i = 0; i < 3; i++)
            tfm[9 + i] = (float)(-(R[i] * t[0] + R[3 + i] * t[1] + R[6 + i] * t[2]));
    }
    return ok;
}

int gto_solve(const float* sums15, int n, float* tfm12) {
    return solve_sums(sums15, n, 0, tfm12);
}

/* ------------------------------------------------------------------------ */
/* secondary structure: MpSecStr.cpp:26-118, MpSecStr.h:218-249              */
static float ss_dst(const float* x, const float* y, const float* z, int i, int j) {
    float dx = x[i] - x[j], dy = y[i] - y[j], dz = z[i] - z[j];
    float a = dx * dx;
    float b = dy * dy;
    float c = dz * dz;
    return sqrtf((a + b) + c);
}
/* Secondary structure of a nucleic-acid chain (MpSecStr.cpp:140-200 and
 * 265-360, MpSecStr.h:163-200): every residue gets '.'; residue y's
 * partner is the residue x, more than 2 positions away and of a
 * complementary base (A-T/U, G-C, G-U), whose C3' distance deviates least
 * from 13.75 A (at most 1.25 A); y and x pair, '(' then ')', when each is
 * the other's partner. */
void gto_secstr_na(int len, const float* x, const float* y, const float* z,
                   const unsigned char* rsd, char* ss) {
    int* partner = (int*)malloc(sizeof(int) * (len > 0 ? len : 1));
    for (int p = 0; p < len; p++) { ss[p] = '.'; partner[p] = -1; }
    for (int yi = 0; yi < len; yi++) {
        char a = (char)rsd[yi];
        float best = 9999.9f;
        int col = -1;
        for (int xi = 0; xi < len; xi++) {
            char b = (char)rsd[xi];
            int cond = ((a == 'T' || a == 'U') && b == 'A') || (a == 'A' && (b == 'T' || b == 'U')) ||
                       (a == 'G' && (b == 'C' || b == 'U')) || ((a == 'C' || a == 'U') && b == 'G');
            if (!cond || abs(xi - yi) <= 2) continue;
            float dev = fabsf(ss_dst(x, y, z, yi, xi) - 13.75f);
            if (1.25f < dev) dev = 9999.9f;
            if (dev < best) { best = dev; col = xi; }
        }
        if (best < 1.5f) partner[yi] = col;
    }
    for (int p = 0; p < len; p++) {
        int q = partner[p];
        if (0 <= q && q < len && p < q && partner[q] == p) { ss[p] = '('; ss[q] = ')'; }
    }
    free(partner);
}

void gto_secstr(int len, const float* x, const float* y, const float* z, char* ss) {
    for (int p = 0; p < len; p++) ss[p] = ' ';
    for (int p = 2; p + 2 < len; p++) {
        float d13 = ss_dst(x, y, z, p - 2, p);
        float d14 = ss_dst(x, y, z, p - 2, p + 1);
        float d15 = ss_dst(x, y, z, p - 2, p + 2);
        float d24 = ss_dst(x, y, z, p - 1, p + 1);
        float d25 = ss_dst(x, y, z, p - 1, p + 2);
        float d35 = ss_dst(x, y, z, p, p + 2);
        float e = 2.1f;
        char s = ' ';
        if (fabsf(d15 - 6.37f) < e && fabsf(d14 - 5.18f) < e && fabsf(d25 - 5.18f) < e &&
            fabsf(d13 - 5.45f) < e && fabsf(d24 - 5.45f) < e && fabsf(d35 - 5.45f) < e)
            s = 'h';
        else {
            e = 1.42f;
            if (fabsf(d15 - 13.0f) < e && fabsf(d14 - 10.4f) < e && fabsf(d25 - 10.4f) < e &&
                fabsf(d13 - 6.1f) < e && fabsf(d24 - 6.1f) < e && fabsf(d35 - 6.1f) < e)
                s = 'e';
            else if (d15 < 8.0f)
                s = 't';
        }
        ss[p] = s;
    }
}

/* ------------------------------------------------------------------------ */
/* pair context                                                              */
typedef struct {
    int lq, lr;
    const float *qx, *qy, *qz, *rx, *ry, *rz;
    const unsigned char *qa, *ra;
    const char *qs, *rs;
    int qmol, rmol;
    int ri;              /* the reference's index in its block */
    /* chunk-level values */
    int qmax, rmax, qmin, rmin;
    const gto_opts* o;
    /* state */
    int flags;
    float grand, best, best0;
    int seedq, seedr;
    int naln;
    int sfndx, sfpos;           /* fragment of the final-phase-1 winner */
    int sfndx_cur, sfpos_cur;
    float tfm_ib[12], tfm_gr[12];
    int *aq, *ar;               /* aligned pairs, forward order */
    float *ad;                  /* constrained: dist2 */
    unsigned char* bt;          /* traceback lq*lr */
    float *h0, *h1;
    float out[GTO_NOUT];
    float err[GTO_NERR];
    float d0, d02, d82, d0fin, d0s;
    /* detailed search: the structures' index trees, the best transform among
     * its refined branches, and the refinement variants (1..95: the three
     * sections' slots) the first DP refinement after it skips (the fragment
     * slots its sorting left without a DP score) */
    const float *qnx, *qny, *qnz, *rnx, *rny, *rnz;
    const int *qnl, *qnr, *qno, *rnl, *rnr, *rno;
    float tfm_2nd[12];
    unsigned vskip[3];
} pairctx;

static void tfm_identity(float* t) { memset(t, 0, 12 * sizeof(float)); t[0] = t[4] = t[8] = 1.f; }

/* positions of k-space: 0 = gapless diagonal from (q0,r0); 1 = aligned pairs */
typedef struct { int mode; int q0, r0; const int *aq, *ar; } kspace;
static inline void kpos(const kspace* s, int k, int* q, int* r) {
    if (s->mode == 0) { *q = s->q0 + k; *r = s->r0 + k; }
    else { *q = s->aq[k]; *r = s->ar[k]; }
}

/* covariance over [k0,k1) (all positions) */
/* covariance over positions [k0,k1); the compensated blocks are the
 * absolute position blocks [32m, 32m+32) of the position space (the first
 * and last ones clipped to the range), so that every pass over a space
 * folds at the same positions whatever range it covers */
static void cov_range(const pairctx* P, const kspace* s, int k0, int k1, float* v) {
    ccacc a; cc_init(&a);
    for (int k = k0; k < k1; k++) {
        int q, r; kpos(s, k, &q, &r);
        cc_add(&a, P->qx[q], P->qy[q], P->qz[q], P->rx[r], P->ry[r], P->rz[r]);
        if ((k + 1) % GTB_BLK == 0) cc_fold(&a);
    }
    cc_final(&a, v);
}
/* covariance over [0,n) of positions with dist2(tfm) <= thr */
static void cov_ext(const pairctx* P, const kspace* s, int n, const float* tfm,
                    float thr, float* v) {
    ccacc a; cc_init(&a);
    int blk = 0;
    for (int k = 0; k < n; k++) {
        int q, r; kpos(s, k, &q, &r);
        float qx = P->qx[q], qy = P->qy[q], qz = P->qz[q];
        float rx = P->rx[r], ry = P->ry[r], rz = P->rz[r];
        float d = dist2_tf(tfm, qx, qy, qz, rx, ry, rz);
        if (d <= thr) cc_add(&a, qx, qy, qz, rx, ry, rz);
        if (++blk == GTB_BLK) { cc_fold(&a); blk = 0; }
    }
    cc_final(&a, v);
}

/* score pass over [0,n); chk: only d<=d82 contribute;
 * m3mode: 0 none, 1 distinct (findfrag), 2 multiset (refinement) */
static float score_pass(const pairctx* P, const kspace* s, int n, const float* tfm,
                        float d02, int chk, float d82, int m3mode, float* m3out) {
    float ss = 0.f, sc = 0.f, sb = 0.f;
    int blk = 0;
    float m1 = LARGEDST, m2 = LARGEDST, m3 = LARGEDST;
    for (int k = 0; k < n; k++) {
        int q, r; kpos(s, k, &q, &r);
        float d = dist2_tf(tfm, P->qx[q], P->qy[q], P->qz[q], P->rx[r], P->ry[r], P->rz[r]);
        if (!chk || d <= d82) sb += d02 / (d02 + d);
        if (m3mode == 2) {
            if (d < m1) { m3 = m2; m2 = m1; m1 = d; }
            else if (d < m2) { m3 = m2; m2 = d; }
            else if (d < m3) m3 = d;
        } else if (m3mode == 1) {
            if (d < m1) { m3 = m2; m2 = m1; m1 = d; }
            else if (d > m1 && d < m2) { m3 = m2; m2 = d; }
            else if (d > m2 && d < m3) m3 = d;
        }
        if (++blk == GTB_BLK) { nfold(&ss, &sc, &sb); blk = 0; }
    }
    nfold(&ss, &sc, &sb);
    if (m3out) *m3out = m3;
    return ss + sc;
}

/* convergence of all 16 fields: MpStageBase.h:244-264 */
static int converged16(const float* a, const float* b) {
    int cnt = 0;
    for (int f = 0; f < 16; f++) {
        float x = a[f], y = b[f];
        float m = fabsf(x) < fabsf(y) ? fabsf(x) : fabsf(y);
        if (fabsf(x - y) < m * RM_CONVEPS) cnt++;
    }
    return cnt >= 16;
}

static int solve_pair(const pairctx* P, const float* v, float* tfm) {
    int n = (int)v[15];
    int swap = P->o->symmetric && (P->lq < P->lr);
    return solve_sums(v, n, swap, tfm);
}

/* ------------------------------------------------------------------------ */
/* stage 1: fragment seed, MpStage1.cpp:289-440 (per offset)                 */
static float findfrag_variant(const pairctx* P, int qpos, int rpos, int n) {
    kspace s = {0, qpos, rpos, NULL, NULL};
    float v[16], tfm[12], m3, best = 0.f;
    float d02s0 = P->d0s * P->d0s;
    cov_range(P, &s, 0, n, v);
    for (int it = 0; it < 3; it++) {
        solve_pair(P, v, tfm);
        int save = (it < 2);
        float sc = score_pass(P, &s, n, tfm, P->d02, 0, 0.f, save ? 1 : 0, &m3);
        if (best < sc) best = sc;
        if (!save) break;
        float d02s = d02s0 + (it == 1 ? 1.0f : 0.0f);
        float dst32;
        if (LARGEDST_CMP < m3 || m3 < d02s || n <= 3) dst32 = d02s;
        else dst32 = d02s + ceilf((m3 - d02s) * 2.0f) * 0.5f;
        cov_ext(P, &s, n, tfm, dst32, v);
        if (v[15] < 1.0f) break;
        if ((int)v[15] == n) break;
    }
    return best;
}

static void stage1_findfrag(pairctx* P) {
    if (P->flags & CONV_LOWTMSC) return;
    int minlenmin = P->qmin < P->rmin ? P->qmin : P->rmin;
    int minalnmin = (minlenmin >> 1) > 5 ? (minlenmin >> 1) : 5;
    int n1 = minalnmin - P->rmax;
    int n2 = P->qmax - minalnmin;
    int step = P->o->stepinit;
    int nsteps = (n2 - n1) / step + 1;
    int prv = (P->lq < P->lr ? P->lq : P->lr) >> 1;
    if (prv < 5) prv = 5;
    float best = 0.f;
    int bq = 0, br = 0;
    for (int si = 0; si < nsteps; si++) {
        int ab = n1 + si * step;
        int qpos = ab > 0 ? ab : 0;
        int rpos = -ab > 0 ? -ab : 0;
        if (P->lq <= qpos || P->lr <= rpos) continue;
        if (P->lq - qpos < prv || P->lr - rpos < prv) continue;
        int n = (P->lq - qpos) < (P->lr - rpos) ? (P->lq - qpos) : (P->lr - rpos);
        float b = findfrag_variant(P, qpos, rpos, n);
        if (b > 0.f && best < b) { best = b; bq = qpos; br = rpos; }
    }
    P->best = best;
    P->seedq = bq;
    P->seedr = br;
}

/* generic refinement loop: MpStage1.cpp:640-700 (and its copies) */
static void refine_loop(const pairctx* P, const kspace* s, int nrange, int kf, int fraglen,
                        float d0, float d02, int chk, float d82, float best_init,
                        float* bestout, float* tfmbest) {
    float v[16], last[16], tfm[12], m3 = LARGEDST, dst32 = LARGEDST;
    float best = best_init;
    float d0s = c_d0s(d0);
    float thr2 = (d0s + 1.0f) * (d0s + 1.0f);
    cov_range(P, s, kf, kf + fraglen, v);
    float prev_tfm[12];
    for (int cit = 0; cit < NMAXCONVIT + 2; cit++) {
        if (cit > 0) {
            cov_ext(P, s, nrange, prev_tfm, (cit < 2) ? dst32 : thr2, v);
            if (converged16(v, last)) break;
        }
        if (v[15] < 1.0f) break;
        memcpy(last, v, sizeof(last));
        solve_pair(P, v, tfm);
        float sc = score_pass(P, s, nrange, tfm, d02, chk, d82, cit < 1 ? 2 : 0, &m3);
        if (cit < 1) {
            float d0sm = d0s - 1.0f;
            float d02s = d0sm * d0sm;
            if (LARGEDST_CMP < m3 || m3 < d02s || nrange <= 3) dst32 = d02s;
            else {
                float t = d0sm + ceilf((sqrtf(m3) - d0sm) * 2.0f) * 0.5f;
                dst32 = t * t;
            }
        }
        if (best < sc) { best = sc; memcpy(tfmbest, tfm, sizeof(tfm)); }
        memcpy(prev_tfm, tfm, sizeof(tfm));
    }
    *bestout = best;
}

/* variant enumeration of the 6-length x step-40 refinement */
static int nlocsteps_refine(const pairctx* P) {
    int maxalnmax = P->qmax < P->rmax ? P->qmax : P->rmax;
    return max_nfrag_steps(maxalnmax, FRAG_STEP, MINFRAGLEN) * FRAG_NSUB;
}

/* RefineFragInit (dpmode 0) and RefineFragDP (dpmode 1) and FinalPhase1
 * (dpmode 2): winner = max score > 0, lowest variant index on ties. */
static void refine_stage(pairctx* P, int dpmode, float d0, float d02, int chk,
                         float best_init, int grandupd, int writefrag) {
    int nloc = nlocsteps_refine(P);
    kspace s;
    int nrange;
    if (dpmode == 0) {
        s.mode = 0; s.q0 = P->seedq; s.r0 = P->seedr; s.aq = s.ar = NULL;
        if (P->lq <= P->seedq || P->lr <= P->seedr) nrange = 0;
        else nrange = (P->lq - P->seedq) < (P->lr - P->seedr) ? (P->lq - P->seedq) : (P->lr - P->seedr);
    } else {
        s.mode = 1; s.aq = P->aq; s.ar = P->ar; s.q0 = s.r0 = 0;
        nrange = P->naln;
    }
    float wbest = 0.f, wtfm[12];
    int wsi = -1, wndx = 0, wpos = 0;
    for (int si = 0; si < nloc && nrange > 0; si++) {
        if (dpmode == 1 && si < 96 && ((P->vskip[si >> 5] >> (si & 31)) & 1u)) continue;
        int sfragfct = si / FRAG_NSUB, sfragndx = si % FRAG_NSUB;
        int fraglen = frag_length(nrange, sfragndx);
        if (fraglen < 1) continue;
        int sfragpos = sfragfct * FRAG_STEP;
        if (nrange + FRAG_STEP <= sfragpos + fraglen) continue;
        int delta = sfragpos + fraglen - nrange;
        int kf = sfragpos - (delta > 0 ? delta : 0);
        float best, tb[12];
        refine_loop(P, &s, nrange, kf, fraglen, d0, d02, chk, P->d82, best_init, &best, tb);
        if (best > 0.f && wbest < best) {
            wbest = best; wsi = si; memcpy(wtfm, tb, sizeof(wtfm));
            wndx = sfragndx; wpos = sfragpos;
        }
    }
    P->best = wbest;
    if (wsi >= 0) memcpy(P->tfm_ib, wtfm, sizeof(wtfm));
    if (writefrag) {
        if (wsi >= 0) { P->sfndx_cur = wndx; P->sfpos_cur = wpos; }
        P->sfndx = P->sfndx_cur; P->sfpos = P->sfpos_cur;
    }
    if (grandupd && P->grand < wbest) {
        P->grand = wbest;
        memcpy(P->tfm_gr, wtfm, sizeof(wtfm));
    }
}

/* Final phase 2: one fragment length (the phase-1 winner's, 0 promoted to 1)
 * at nf positions around the phase-1 position (MpStageFin.cpp:270-480), or,
 * with full = 1 (--refinement 4), every fragment length at each position,
 * variant index = position factor * 6 + length index, no promotion
 * (covariance_fin_dp_refn_complete.cu:464-630, custage_fin.cu:272-275,344). */
static void final_phase2(pairctx* P, int full) {
    int maxalnmax = P->qmax < P->rmax ? P->qmax : P->rmax;
    int nf = 2 * maxalnmax < FIN_MAXNPOS ? 2 * maxalnmax : FIN_MAXNPOS;
    kspace s = {1, 0, 0, P->aq, P->ar};
    int n = P->naln;
    float wbest = 0.f, wtfm[12];
    int wsi = -1;
    int nsi = full ? nf * FRAG_NSUB : nf;
    for (int si = 0; si < nsi; si++) {
        int sfragfct = full ? si / FRAG_NSUB : si;
        int sfragndx = full ? si % FRAG_NSUB : P->sfndx;
        int sfragpos = P->sfpos;
        if (!full && sfragndx == 0) sfragndx++;
        sfragpos += (sfragfct - (nf >> 1));
        int fraglen = frag_length(n, sfragndx);
        if (fraglen < 1) continue;
        if (sfragpos < 0 || n + 1 <= sfragpos + fraglen) continue;
        float best, tb[12];
        refine_loop(P, &s, n, sfragpos, fraglen, P->d0, P->d02, 1, P->d82, -1.0f, &best, tb);
        if (best > 0.f && wbest < best) { wbest = best; wsi = si; memcpy(wtfm, tb, sizeof(wtfm)); }
    }
    P->best = wbest;
    if (wsi >= 0) memcpy(P->tfm_ib, wtfm, sizeof(wtfm));
    if (P->grand < wbest) { P->grand = wbest; memcpy(P->tfm_gr, wtfm, sizeof(wtfm)); }
}

/* ------------------------------------------------------------------------ */
/* DP: MpDPHub.cpp:72-346 (plain) and :686-940 (grand tfm + SS)            */
static void dp_run(pairctx* P, const float* tfm, int gap0, float gcost, int usess,
                   float d02) {
    int lq = P->lq, lr = P->lr;
    float* prev = P->h0;   /* row i-1 */
    float* cur = P->h1;
    for (int j = 0; j < lr; j++) prev[j] = 0.f;
    for (int i = 0; i < lq; i++) {
        float tx, ty, tz;
        xform(tfm, P->qx[i], P->qy[i], P->qz[i], &tx, &ty, &tz);
        char qs = usess ? P->qs[i] : 0;
        float left = 0.f;          /* H[i][j-1], boundary 0 */
        for (int j = 0; j < lr; j++) {
            float dx = tx - P->rx[j], dy = ty - P->ry[j], dz = tz - P->rz[j];
            float d = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
            float v = d02 / (d02 + d);
            if (usess) v += (float)(qs == P->rs[j]) * 0.5f;
            float dg = (j > 0) ? prev[j - 1] : 0.f;
            v += gap0 ? dg : fabsf(dg);
            int bk = BT_DIAG;
            float l = left;
            if (!gap0 && l < 0.f) l = gcost - l;
            if (v < l) { v = l; bk = BT_LEFT; }
            float u = prev[j];
            if (!gap0 && u < 0.f) u = gcost - u;
            if (v < u) { v = u; bk = BT_UP; }
            float w = (gap0 || bk != BT_DIAG) ? v : -v;
            cur[j] = w;
            left = w;
            P->bt[(size_t)i * lr + j] = (unsigned char)bk;
        }
        float* t = prev; prev = cur; cur = t;
    }
}

/* DP of the --add-search-by-ss stage (dpssw_btck.cu:280-330,
 * MpDPHub.cpp:985-1210): no transform; a cell scores 1 for equal secondary
 * structure plus 0.2 x the Gonnet score of the residue pair.  The gap cost
 * is paid once, leaving a cell reached diagonally (gap extension free):
 * such a cell stores its value plus DPSS_C (a large negative offset, so the
 * stored value is rounded to a multiple of 1/8) and a reader takes the offset
 * off again; the matrix border reads as a diagonal cell of value 0. */
#define DPSS_C (-1048576.0f)
#define DPSS_CMP (-524288.0f)
static float g_gonnet[GTB_GONNET_NA * GTB_GONNET_NA];

static float gonnet_score(unsigned char a, unsigned char b) {
    if ('A' <= a && a <= 'Z' && 'A' <= b && b <= 'Z') return g_gonnet[(a - 'A') * GTB_GONNET_NA + (b - 'A')];
    return 0.0f;
}

static void dp_ss_run(pairctx* P, float gcost) {
    int lq = P->lq, lr = P->lr;
    float* prev = P->h0;   /* row i-1 */
    float* cur = P->h1;
    for (int j = 0; j < lr; j++) prev[j] = DPSS_C;
    for (int i = 0; i < lq; i++) {
        char qs = P->qs[i];
        unsigned char qa = P->qa[i];
        float left = DPSS_C;
        for (int j = 0; j < lr; j++) {
            float v = fmaf(gonnet_score(qa, P->ra[j]), 0.2f, (float)(qs == P->rs[j]));
            float dg = (i > 0 && j > 0) ? prev[j - 1] : DPSS_C;
            if (dg < DPSS_CMP) dg = dg - DPSS_C;
            v = v + dg;
            int bk = BT_DIAG;
            float l = left;
            if (l < DPSS_CMP) l = (gcost + l) - DPSS_C;
            if (v < l) { v = l; bk = BT_LEFT; }
            float u = prev[j];
            if (u < DPSS_CMP) u = (gcost + u) - DPSS_C;
            if (v < u) { v = u; bk = BT_UP; }
            float w = (bk == BT_DIAG) ? v + DPSS_C : v;
            cur[j] = w;
            left = w;
            P->bt[(size_t)i * lr + j] = (unsigned char)bk;
        }
        float* t = prev; prev = cur; cur = t;
    }
}

/* --pre-similarity (MpStage1.cpp:175-248, PMBatchStrData.inl:37-95): the pair
 * passes when some diagonal, every 2nd one at least 20 residues from either
 * end, has an ungapped run of residue pairs whose Gonnet scores sum to the
 * threshold or more.  The diagonals are numbered over the block's longest
 * query and reference; diagonal di starts at query position 2*di, or, past
 * the query's last admissible start, at reference position
 * ((2*di - (lq - 20)) rounded down to even) + 2. */
#define PRESIM_EDGE 20
#define PRESIM_STEP 2
static int presim_pass(const pairctx* P, float thr) {
    int ql = P->lq, rl = P->lr;
    int ndiag = (P->qmax + P->rmax - 2 * PRESIM_EDGE) >> 1;
    for (int di = 0; di < ndiag; di++) {
        int qp = di * PRESIM_STEP, rp = 0;
        if (ql - PRESIM_EDGE <= qp) {
            rp = ((qp - (ql - PRESIM_EDGE)) & ~1) + PRESIM_STEP;
            qp = 0;
        }
        if (ql - PRESIM_EDGE <= qp || rl - PRESIM_EDGE <= rp) continue;
        int n1 = ql - qp < rl ? ql - qp : rl, n2 = rl - rp < ql ? rl - rp : ql;
        int n = n1 < n2 ? n1 : n2;
        float s = 0.f, mn = 0.f, best = 0.f;
        for (int k = 0; k < n; k++) {
            s = s + gonnet_score(P->qa[qp + k], P->ra[rp + k]);
            mn = s < mn ? s : mn;
            float loc = s - mn;
            best = loc > best ? loc : best;
        }
        if (thr <= best) return 1;
    }
    return 0;
}

/* unconstrained traceback: MpDPHub.cpp:1515-1660 */
static void btck_matched(pairctx* P) {
    int y = P->lq - 1, x = P->lr - 1, n = 0;
    while (x >= 0 && y >= 0) {
        int b = P->bt[(size_t)y * P->lr + x];
        if (b == BT_UP) { y--; continue; }
        if (b == BT_LEFT) { x--; continue; }
        P->aq[n] = y; P->ar[n] = x; n++;
        x--; y--;
    }
    /* reverse to forward order */
    for (int i = 0, j = n - 1; i < j; i++, j--) {
        int t = P->aq[i]; P->aq[i] = P->aq[j]; P->aq[j] = t;
        t = P->ar[i]; P->ar[i] = P->ar[j]; P->ar[j] = t;
    }
    P->naln = n;
}

/* constrained traceback: keep d2 <= d82 under the grand tfm */
static void btck_constrained(pairctx* P) {
    int y = P->lq - 1, x = P->lr - 1, n = 0;
    while (x >= 0 && y >= 0) {
        int b = P->bt[(size_t)y * P->lr + x];
        if (b == BT_UP) { y--; continue; }
        if (b == BT_LEFT) { x--; continue; }
        float d = dist2_tf(P->tfm_gr, P->qx[y], P->qy[y], P->qz[y], P->rx[x], P->ry[x], P->rz[x]);
        if (d <= P->d82) { P->aq[n] = y; P->ar[n] = x; P->ad[n] = d; n++; }
        x--; y--;
    }
    for (int i = 0, j = n - 1; i < j; i++, j--) {
        int t = P->aq[i]; P->aq[i] = P->aq[j]; P->aq[j] = t;
        t = P->ar[i]; P->ar[i] = P->ar[j]; P->ar[j] = t;
        float f = P->ad[i]; P->ad[i] = P->ad[j]; P->ad[j] = f;
    }
    P->naln = n;
}

/* DP + traceback with the iteration-best transform (DPRefine body) */
static int dp_skip_plain(const pairctx* P) {
    return (P->flags & CONV_LOWTMSC) || (P->flags & CONV_SCOREDP);
}

/* tfm1 (may be NULL): the transform of the first DP instead of the
 * iteration-best one (WRKMEMTM1, MpStage1.cpp:489-493) */
static void dprefine_t(pairctx* P, int gap0, int prescreen, int maxit, const float* tfm1) {
    float gcost = gap0 ? 0.0f : -0.6f;
    for (int dpi = 0; dpi < maxit; dpi++) {
        if (!dp_skip_plain(P)) {
            dp_run(P, (tfm1 && dpi == 0) ? tfm1 : P->tfm_ib, gap0, gcost, 0, P->d02);
            btck_matched(P);
        } else P->naln = 0;
        if (P->flags) P->best = 0.f;   /* variants skipped: slot bests were reset */
        else refine_stage(P, 1, P->d0, P->d02, 1, 0.f, 1, 0);
        if (0 < dpi && !(P->flags & (CONV_SCOREDP | CONV_LOWTMSC)) &&
            fabsf(P->best - P->best0) < SCORE_CONVEPS)
            P->flags |= CONV_SCOREDP;
        if (dpi + 1 < maxit && !(P->flags & (CONV_SCOREDP | CONV_LOWTMSC)))
            P->best0 = P->best;
        if (prescreen && maxit <= dpi + 1 && 0.0f < P->o->prescore) {
            int ml = P->lq < P->lr ? P->lq : P->lr;
            if (P->grand < P->o->prescore * (float)ml) P->flags |= CONV_LOWTMSC;
        }
    }
    /* InitScoresKernel<INITOPT_CONVFLAG_SCOREDP> over every slot
     * (MpStage1.cpp:510): the pair's flag and the fragment slots' flags */
    P->flags &= ~CONV_SCOREDP;
    P->vskip[0] = P->vskip[1] = P->vskip[2] = 0u;
}

static void dprefine(pairctx* P, int gap0, int prescreen, int maxit) {
    dprefine_t(P, gap0, prescreen, maxit, NULL);
}

/* ------------------------------------------------------------------------ */
/* Spatial-index detailed search: MpStageFrg3::Run (MpStageFrg3.h:80-115,     */
/* MpStageFrg3.cpp:35-469), one pair as if alone in its chunk and processed  */
/* by one thread (the reference's fragment slot of a scored configuration is */
/* its thread's running count of them; its memory alignment of the local    */
/* score matrix follows the chunk layout).                                   */
#define FRG3_NTOP 32            /* CUS1_TBSP_DPSCORE_TOP_N */
#define FRG3_NSEC 3             /* CUS1_TBSP_DPSCORE_TOP_N_MAX_CONFIGS: slot sections */
#define FRG3_LENTHR 150         /* MpStageFrg3.cpp:48 */
#define FRG3_MAXVISIT 64        /* CUSF_TBSP_INDEX_SCORE_MAXDEPTH */
#define FRG3_HASH 512           /* CUSF_TBSP_INDEX_SCORE_POSLIMIT2 */
#define FRG3_SIMROWS 96         /* MPSF_TBSP_LOCAL_SIMILARITY_YDIM x 3 */
#define FRG3_SIMCOLS 128        /* MPSF_TBSP_LOCAL_SIMILARITY_XDIM */
#define FRG3_MAXSTACK 17
#define FRG3_SSDST2 64.0f       /* SS-matched neighbour farther than 8 A: none */

/* local alignment by secondary structure (ExecDPSSLocal128xKernel,
 * MpDPHub.cpp:1256-1480): a cell scores +1 for equal, -1 for different SS,
 * floored at 0 (STOP); gaps cost gcost; the byte kept per cell is the
 * truncated score rounded down to a multiple of 4 (mod 256) with the
 * direction in its two low bits */
static void frg3_localdp(pairctx* P, float gcost, unsigned char* m) {
    int lq = P->lq, lr = P->lr;
    float* prev = P->h0;
    float* cur = P->h1;
    for (int j = 0; j < lr; j++) prev[j] = 0.f;
    for (int i = 0; i < lq; i++) {
        char qs = P->qs[i];
        float left = 0.f;
        for (int j = 0; j < lr; j++) {
            float v = (float)((qs == P->rs[j]) * 2) - 1.0f;
            v = v + ((j > 0) ? prev[j - 1] : 0.f);
            int bk = BT_DIAG;
            if (v < 0.f) { v = 0.f; bk = BT_STOP; }
            float l = left + gcost;
            if (v < l) { v = l; bk = BT_LEFT; }
            float u = prev[j] + gcost;
            if (v < u) { v = u; bk = BT_UP; }
            cur[j] = v;
            left = v;
            m[(size_t)i * lr + j] = (unsigned char)((((unsigned)v) & 0xfcu) | (unsigned)bk);
        }
        float* t = prev; prev = cur; cur = t;
    }
}

/* fragment lengths (GetNAlnPoss_frg, covariancebase.h:93-110) */
static int frg3_fraglen(int lq, int lr, int fi, int seedrule) {
    int minlen = lq < lr ? lq : lr;
    int half = minlen >> 1;
    if (seedrule) return seedrule < half ? seedrule : half;
    if (fi == 0) {
        int leno3 = (int)((float)minlen * (1.0f / 3.0f));
        if (leno3 < 1) leno3 = 1;
        return leno3 < 20 ? leno3 : 20;
    }
    return half < 100 ? half : 100;
}

/* position step of the configurations (GetFragStepSize_frg_*,
 * covariancebase.h:22-84) */
static int frg3_step(int depth, int len) {
    int leno3 = (int)((float)len * (1.0f / 3.0f));
    if (leno3 < 1) leno3 = 1;
    int small = leno3 < 15 ? leno3 : 15;
    if (depth == 0) return len > 150 ? 15 : small;
    if (depth == 1) return len > 150 ? 23 : small;
    int med = len > 250 ? 45 : len > 200 ? 35 : len > 150 ? 25 : small;
    return depth == 2 ? med : 2 * med;
}

/* The local similarity test of a configuration (CalcLocalSimilarity2_frg2,
 * MpStageFrg3.h:327-415): the largest score byte over 96 rows from qrypos and
 * up to 128 columns from rfnpos (rounded up to a multiple of 4, as the
 * 4-byte reads of a structure starting on such a boundary) must reach the
 * fragment length x the trigger fraction. */
static int frg3_similar(const pairctx* P, const unsigned char* m, int qrypos, int rfnpos,
                        int fl, float thr) {
    if (P->lq < qrypos + fl) fl = P->lq - qrypos;
    if (P->lr < rfnpos + fl) fl = P->lr - rfnpos;
    int pidelta = (P->lr - 3 - rfnpos) & ~3;
    if (pidelta > FRG3_SIMCOLS) pidelta = FRG3_SIMCOLS;
    int pibeg = (rfnpos + 3) & ~3;
    unsigned maxg = 0;
    for (int ii = 0; qrypos + ii < P->lq && ii < FRG3_SIMROWS; ii++) {
        const unsigned char* row = m + (size_t)(qrypos + ii) * P->lr;
        for (int pi = pibeg; pi < pibeg + pidelta; pi++) {
            unsigned v = row[pi] & 0xfcu;
            if (v > maxg) maxg = v;
        }
    }
    return !((float)maxg < (float)fl * thr);
}

/* Sum over 32 values in the order of a warp's xor-shuffle reduction
 * (offsets 16, 8, 4, 2, 1); every lane ends with this value. */
static float tree32(const float* t) {
    float a[32];
    memcpy(a, t, sizeof(a));
    for (int off = 16; off > 0; off >>= 1) {
        float b[32];
        for (int k = 0; k < 32; k++) b[k] = a[k] + a[k ^ off];
        memcpy(a, b, sizeof(a));
    }
    return a[0];
}

/* Covariance sums over position slots 0..n-1 (pairs (pq[k], pr[k]); a
 * negative index: no pair): slots in blocks of 32, each block summed by
 * tree32 per field and folded into Neumaier totals in block order. */
static void frg3_cov(const pairctx* P, const int* pq, const int* pr, int n, float* v) {
    float s[15], c[15], b[15];
    for (int f = 0; f < 15; f++) s[f] = c[f] = 0.f;
    int cnt = 0;
    for (int b0 = 0; b0 < n; b0 += 32) {
        float t[15][32];
        for (int k = 0; k < 32; k++) {
            int i = b0 + k;
            int ok = i < n && pq[i] >= 0 && pr[i] >= 0;
            float qx = ok ? P->qx[pq[i]] : 0.f, qy = ok ? P->qy[pq[i]] : 0.f, qz = ok ? P->qz[pq[i]] : 0.f;
            float rx = ok ? P->rx[pr[i]] : 0.f, ry = ok ? P->ry[pr[i]] : 0.f, rz = ok ? P->rz[pr[i]] : 0.f;
            t[0][k] = qx * rx; t[1][k] = qx * ry; t[2][k] = qx * rz;
            t[3][k] = qy * rx; t[4][k] = qy * ry; t[5][k] = qy * rz;
            t[6][k] = qz * rx; t[7][k] = qz * ry; t[8][k] = qz * rz;
            t[9][k] = qx; t[10][k] = qy; t[11][k] = qz;
            t[12][k] = rx; t[13][k] = ry; t[14][k] = rz;
            cnt += ok;
        }
        for (int f = 0; f < 15; f++) { b[f] = tree32(t[f]); nfold(&s[f], &c[f], &b[f]); }
    }
    for (int f = 0; f < 15; f++) v[f] = s[f] + c[f];
    v[15] = (float)cnt;
}

/* Seed positions from the local alignment (CalcCCMatricesLocallyAligned_
 * Complete, MpStage1.h:395-470): of 4 evenly spaced cells, the first with
 * the largest score byte; the local alignment traced back from it within the
 * rectangle from (qrypos, rfnpos).  Returns the aligned pairs in increasing
 * order, or 0 when too few. */
static int frg3_seed_local(const pairctx* P, const unsigned char* m, int trig, int fraglen,
                           int qrypos, int rfnpos, int* pq, int* pr) {
    int lq = P->lq, lr = P->lr;
    if (lq < qrypos + fraglen && lr < rfnpos + fraglen)
        fraglen = (lq - qrypos) > (lr - rfnpos) ? (lq - qrypos) : (lr - rfnpos);
    fraglen >>= 2;
    int y = qrypos, x = rfnpos;
    float vr = 0.f;
    for (int f = 0; f < 4; f++) {
        int yt = qrypos + (f + 1) * fraglen, xt = rfnpos + (f + 1) * fraglen;
        if (yt > lq - 1) yt = lq - 1;
        if (xt > lr - 1) xt = lr - 1;
        float vrt = (float)(m[(size_t)yt * lr + xt] & 0xfcu);
        if (vr < vrt) { vr = vrt; y = yt; x = xt; }
    }
    int n = 0;
    while (y >= qrypos && x >= rfnpos) {
        int b = m[(size_t)y * lr + x] & 3;
        if (b == BT_STOP) break;
        if (b == BT_UP) { y--; continue; }
        if (b == BT_LEFT) { x--; continue; }
        pq[n] = y; pr[n] = x; n++;
        x--; y--;
    }
    int minf = fraglen < 16 ? fraglen : 16;
    if (n < 1 || (trig && n < minf)) return 0;
    for (int i = 0, j = n - 1; i < j; i++, j--) {
        int t = pq[i]; pq[i] = pq[j]; pq[j] = t;
        t = pr[i]; pr[i] = pr[j]; pr[j] = t;
    }
    return n;
}

/* Nearest neighbour of (px, py, pz) in a structure's 3-d tree (NNByIndex*,
 * MpStageFrg3.h:1270-1440): depth-first with a bounded stack, at most 64
 * nodes visited; with ss, only residues of that secondary structure count
 * and one farther than 8 A is none.  Returns the residue index or -1. */
static int frg3_nn(const float* nx, const float* ny, const float* nz, const int* nl,
                   const int* nr, const int* no, const char* sss, int len, int ssfilt, char ss,
                   float px, float py, float pz, int stacksize) {
    int stk_node[FRG3_MAXSTACK], stk_dim[FRG3_MAXSTACK];
    float stk_diff[FRG3_MAXSTACK];
    int sp = 0, nvisited = 0, best = -1, root = len >> 1, dim = 0;
    float bestd = 9.9e6f;
    while (0 < sp || 0 <= root) {
        if (0 <= root) {
            nvisited++;
            if (FRG3_MAXVISIT <= nvisited) break;
            int org = no[root];
            float x = nx[root], y = ny[root], z = nz[root];
            float dx = x - px, dy = y - py, dz = z - pz;
            float d2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
            if ((best < 0 || d2 < bestd) && (!ssfilt || sss[org] == ss)) {
                bestd = d2;
                best = ssfilt ? org : root;
            }
            if (bestd == 0.0f) break;
            float diffc = dim == 0 ? dx : (dim == 1 ? dy : dz);
            if (2 < ++dim) dim = 0;
            if (sp < stacksize) { stk_node[sp] = root; stk_dim[sp] = dim; stk_diff[sp] = diffc; sp++; }
            root = (0.0f < diffc) ? nl[root] : nr[root];
        } else {
            int cond = 0;
            float diffc = 0.f;
            while (0 < sp && !cond) {
                sp--;
                root = stk_node[sp]; dim = stk_dim[sp]; diffc = stk_diff[sp];
                cond = diffc * diffc < bestd;
            }
            if (!cond) break;
            root = (0.0f < diffc) ? nr[root] : nl[root];
        }
    }
    if (ssfilt) return FRG3_SSDST2 < bestd ? -1 : best;
    return 0 <= best ? no[best] : -1;
}

/* Neighbours over the window of the shorter structure
 * (ProduceAlignmentUsingIndex2Reference/Query, MpStageFrg3.h:500-680): the
 * window of up to `window` positions about the configuration's position of
 * the shorter structure is moved by tfm (which maps the shorter onto the
 * longer structure) and each position paired with its nearest residue of the
 * longer one; a neighbour at residue 0 or none leaves the slot empty.
 * Fills pq/pr per window slot (-1: empty); returns the window length. */
static int frg3_window(const pairctx* P, const float* tfm, int ssfilt, int window, int qrypos,
                       int rfnpos, int stacksize, int* pq, int* pr) {
    int lq = P->lq, lr = P->lr;
    if (lq < lr) {
        int fl = lr < window ? lr : window;
        int qp = qrypos - (fl >> 1); if (qp < 0) qp = 0;
        int ql = qp + fl < lq ? qp + fl : lq;
        qp = ql - fl; if (qp < 0) qp = 0;
        for (int pi = 0; pi < ql - qp; pi++) {
            int q = qp + pi;
            float x, y, z;
            xform(tfm, P->qx[q], P->qy[q], P->qz[q], &x, &y, &z);
            int r = frg3_nn(P->rnx, P->rny, P->rnz, P->rnl, P->rnr, P->rno, P->rs, lr, ssfilt,
                            P->qs[q], x, y, z, stacksize);
            pq[pi] = q;
            pr[pi] = r > 0 ? r : -1;
        }
        return ql - qp;
    }
    int fl = lq < window ? lq : window;
    int rp = rfnpos - (fl >> 1); if (rp < 0) rp = 0;
    int rl = rp + fl < lr ? rp + fl : lr;
    rp = rl - fl; if (rp < 0) rp = 0;
    for (int pi = 0; pi < rl - rp; pi++) {
        int r = rp + pi;
        float x, y, z;
        xform(tfm, P->rx[r], P->ry[r], P->rz[r], &x, &y, &z);
        int q = frg3_nn(P->qnx, P->qny, P->qnz, P->qnl, P->qnr, P->qno, P->qs, lq, ssfilt,
                        P->rs[r], x, y, z, stacksize);
        pq[pi] = q > 0 ? q : -1;
        pr[pi] = r;
    }
    return rl - rp;
}

/* Order-dependent score of the window's neighbour pairs
 * (CalcScoresUnrl_SWFTscanProgressive_Complete, MpStageFrg3.h:760-850): over
 * the first `cnt` window slots (cnt = the number of non-empty ones), each
 * pair extends the best chain of earlier-partnered pairs kept in a 512-entry
 * table hashed by partner index. */
static float frg3_progressive(const pairctx* P, const float* tfm, const int* pq, const int* pr,
                              int cnt, int partner_is_r) {
    float omax[FRG3_HASH], ondx[FRG3_HASH];
    for (int i = 0; i < FRG3_HASH; i++) { omax[i] = 0.f; ondx[i] = -1.f; }
    for (int pi = 0; pi < cnt; pi++) {
        if (pq[pi] < 0 || pr[pi] < 0) continue;
        float d = dist2_tf(tfm, P->qx[pq[pi]], P->qy[pq[pi]], P->qz[pq[pi]],
                           P->rx[pr[pi]], P->ry[pr[pi]], P->rz[pr[pi]]);
        float sco = P->d02 / (P->d02 + d);
        float qnx = (float)(partner_is_r ? pr[pi] : pq[pi]);
        if (sco <= 0.f) continue;
        float max1 = 0.f;
        for (int ni = 0; ni < FRG3_HASH; ni++)
            if (ondx[ni] < qnx && max1 < omax[ni]) max1 = omax[ni];
        int c = (int)qnx & (FRG3_HASH - 1);
        float st = ondx[c], ss = omax[c], nsc = max1 + sco;
        int half2nd = pi > (cnt >> 1);
        if (st < 0.f || (st == qnx && ss < nsc) || ((half2nd && st < qnx) || (!half2nd && qnx < st))) {
            ondx[c] = qnx;
            omax[c] = nsc;
        }
    }
    float mx = 0.f;
    for (int i = 0; i < FRG3_HASH; i++) if (mx < omax[i]) mx = omax[i];
    return mx;
}

/* GAP0 DP score without traceback (ExecDPScore128xKernel,
 * MpDPHub.cpp:389-645): the value of the last cell */
static float frg3_dpscore(pairctx* P, const float* tfm) {
    int lq = P->lq, lr = P->lr;
    float* prev = P->h0;
    float* cur = P->h1;
    for (int j = 0; j < lr; j++) prev[j] = 0.f;
    for (int i = 0; i < lq; i++) {
        float tx, ty, tz;
        xform(tfm, P->qx[i], P->qy[i], P->qz[i], &tx, &ty, &tz);
        float left = 0.f;
        for (int j = 0; j < lr; j++) {
            float dx = tx - P->rx[j], dy = ty - P->ry[j], dz = tz - P->rz[j];
            float d = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
            float v = P->d02 / (P->d02 + d);
            v += (j > 0) ? prev[j - 1] : 0.f;
            if (v < left) v = left;
            if (v < prev[j]) v = prev[j];
            cur[j] = v;
            left = v;
        }
        float* t = prev; prev = cur; cur = t;
    }
    return prev[lr - 1];
}

static int frg3_stacksize(int lq, int lr) {
    int L = lq > lr ? lq : lr, b = 0;
    while ((1 << b) < L) b++;          /* ceil(log2 L) */
    b += 1;
    return b < FRG3_MAXSTACK ? b : FRG3_MAXSTACK;
}

/* the stage for one pair (runs when the pair is not filtered out) */
static void frg3_stage(pairctx* P) {
    const gto_opts* o = P->o;
    int lq = P->lq, lr = P->lr;
    float thr = (float)o->trigger / 100.0f;
    int seedrule = o->seedrule;
    int mx = lq > lr ? lq : lr;
    int* pq = (int*)malloc(sizeof(int) * (size_t)(mx + o->window + 8));
    int* pr = (int*)malloc(sizeof(int) * (size_t)(mx + o->window + 8));
    unsigned char* m = P->bt;          /* the local score matrix; DP scores below keep it */
    if (0.0f < thr || seedrule) frg3_localdp(P, o->gapcost, m);

    /* the slots of the configuration sections: section 0 takes every scored
     * configuration; at --depth 1 and 0 sections 1 and 2 take those on every
     * second / third grid row and column of a structure longer than 150
     * (sec2met / sec3met, MpStageFrg3.cpp:204-212), in the same slot */
    const int nsec = o->depth <= 0 ? 3 : (o->depth <= 1 ? 2 : 1);
    float sbest[FRG3_NSEC][FRG3_NTOP], stfm[FRG3_NSEC][FRG3_NTOP][12];
    for (int s = 0; s < FRG3_NSEC; s++)
        for (int k = 0; k < FRG3_NTOP; k++) sbest[s][k] = 0.f;
    int nscored = 0;
    int qstep = frg3_step(o->depth, lq), rstep = frg3_step(o->depth, lr);
    int minn = o->depth == 3 ? 5 : 10;
    int nsy = lq / qstep + 1; if (nsy < minn) nsy = minn;
    int nsx = lr / rstep + 1; if (nsx < minn) nsx = minn;
    int stacksize = frg3_stacksize(lq, lr);
    int f0 = frg3_fraglen(lq, lr, 0, 0), f1 = frg3_fraglen(lq, lr, 1, 0);
    int nfr = seedrule ? 1 : 2;
    for (int ys = 0; ys < nsy; ys++)
    for (int xs = 0; xs < nsx; xs++) {
        int qrypos = ys * qstep, rfnpos = xs * rstep;
        int secmet[FRG3_NSEC];
        secmet[0] = 1;
        secmet[1] = o->depth <= 1 && (lq <= FRG3_LENTHR || (ys & 1) == 0) &&
                    (lr <= FRG3_LENTHR || (xs & 1) == 0);
        secmet[2] = o->depth <= 0 && (lq <= FRG3_LENTHR || ys % 3 == 0) &&
                    (lr <= FRG3_LENTHR || xs % 3 == 0);
        /* CalcLocalSimilarity2_frg2: flags of the two fragment lengths */
        if (lq < qrypos + f0 || lr < rfnpos + f0 || f0 < 1) continue;
        int conv1 = (lq < qrypos + f1 || lr < rfnpos + f1 || f1 < 1);
        if (0.0f < thr && !frg3_similar(P, m, qrypos, rfnpos, f1, thr)) continue;
        for (int fi = 0; fi < nfr; fi++) {
            if (fi == 1 && conv1) continue;
            int fraglen = fi == 0 ? f0 : f1;
            if (lq < qrypos + fraglen || lr < rfnpos + fraglen) continue;
            float v[16], tfm[12];
            int n;
            if (seedrule) {
                n = frg3_seed_local(P, m, o->trigger > 0, frg3_fraglen(lq, lr, fi, seedrule),
                                    qrypos, rfnpos, pq, pr);
            } else {
                for (int k = 0; k < fraglen; k++) { pq[k] = qrypos + k; pr[k] = rfnpos + k; }
                n = fraglen;
            }
            if (n < 1) continue;
            frg3_cov(P, pq, pr, n, v);
            if (v[15] < 1.0f) continue;
            /* towards the longer structure (CalcTfmMatrices_DynamicOrientation_Complete) */
            solve_sums(v, (int)v[15], lq < lr ? 0 : 2, tfm);
            for (int it = 0; it < 2; it++) {
                int cw = frg3_window(P, tfm, it == 0, o->window, qrypos, rfnpos, stacksize, pq, pr);
                frg3_cov(P, pq, pr, cw, v);
                if (v[15] < 1.0f) continue;
                if (it == 0) { solve_sums(v, (int)v[15], lq < lr ? 0 : 2, tfm); continue; }
                solve_sums(v, (int)v[15], 0, tfm);
                float sc = frg3_progressive(P, tfm, pq, pr, (int)v[15], lq < lr);
                int slot = nscored % FRG3_NTOP;
                nscored++;
                /* SaveBestScoreAndTM_Complete and Save2ndryScoreAndTM_Complete
                 * (MpStageFrg3.h:887-915): a positive score above the slot's */
                for (int s = 0; s < nsec; s++)
                    if (secmet[s] && 0.0f < sc && sbest[s][slot] < sc) {
                        sbest[s][slot] = sc;
                        memcpy(stfm[s][slot], tfm, sizeof(tfm));
                    }
            }
        }
    }
    /* DP scores of the slots' transforms (SaveTopNScoresAndTMsAmong(Secondary)
     * Bests with one thread keep the slots; ExecDPScore128xKernel skips empty
     * ones), then per section the slots by DP score, larger first, lower slot
     * first on ties (SortBestDPscoresAndTMsAmongDPswifts, MpStageFrg3.h:
     * 1150-1250): a slot rank without a score flags refinement variant
     * section * 32 + rank, section 0's first rank being the pair's flag */
    float dps[FRG3_NSEC][FRG3_NTOP];
    int order[FRG3_NSEC][FRG3_NTOP];
    unsigned vskip[3] = {0u, 0u, 0u};   /* in force only in the DP refinement after the branches */
    for (int s = 0; s < nsec; s++) {
        for (int k = 0; k < FRG3_NTOP; k++) {
            dps[s][k] = 0.0f < sbest[s][k] ? frg3_dpscore(P, stfm[s][k]) : 0.0f;
            order[s][k] = k;
        }
        for (int a = 1; a < FRG3_NTOP; a++) {
            int k = order[s][a], b = a - 1;
            while (b >= 0 && dps[s][order[s][b]] < dps[s][k]) { order[s][b + 1] = order[s][b]; b--; }
            order[s][b + 1] = k;
        }
        for (int r = s == 0 ? 1 : 0; r < FRG3_NTOP; r++)
            if (!(0.0f < dps[s][order[s][r]])) vskip[s] |= 1u << r;
    }
    /* the pair's flag is section 0's first slot's (MpStageFrg3.h:1210-1225) */
    P->flags = 0.0f < dps[0][order[0][0]] ? 0 : CONV_SCOREDP;
    /* the branches, section by section (Refine_tfmaltconfig,
     * MpStageFrg3.cpp:425-467); at --depth 1 and 0 each branch's refinement
     * is followed by one more DP under its iteration-best transform and a
     * refinement of that alignment */
    float best2 = 0.f;
    int nbr = o->nbranches < FRG3_NTOP ? o->nbranches : FRG3_NTOP;
    for (int rci = 0; rci < nsec * nbr; rci++) {
        int s = rci / nbr, k = order[s][rci % nbr];
        int valid = 0.0f < dps[s][k];
        for (int pass = 0; pass < (o->depth <= 1 ? 2 : 1); pass++) {
            if (!(P->flags & (CONV_LOWTMSC | CONV_SCOREDP)) && (valid || pass == 1)) {
                float t[12];
                memcpy(t, pass == 0 ? stfm[s][k] : P->tfm_ib, sizeof(t));
                dp_run(P, t, 1, 0.0f, 0, P->d02);
                btck_matched(P);
            } else P->naln = 0;
            if (P->flags) P->best = 0.f;
            else refine_stage(P, 1, P->d0, P->d02, 1, 0.f, 1, 0);
            /* the best branch's result (SECONDARYUPDATE, MpStageBase.h:1250-1280):
             * unconditional for the first branch */
            if (rci == 0 || best2 < P->best) {
                best2 = P->best;
                memcpy(P->tfm_2nd, P->tfm_ib, sizeof(P->tfm_ib));
            }
        }
    }
    free(pq);
    free(pr);
    /* DP refinement from the best branch, with a gap cost and without
     * (MpStageFrg3.h:108-112); the first one skips the fragment variants of
     * the slots the sorting left empty */
    memcpy(P->vskip, vskip, sizeof(vskip));
    dprefine_t(P, 0, 0, 2, P->tfm_2nd);
    dprefine(P, 1, 0, 2);
}

/* ------------------------------------------------------------------------ */
/* production scores: MpStageFin.cpp:747-1000 and :1310-1525                 */
typedef struct { float best, gbest; float tfm[12]; int ndx, pos; int si; } prodwin;

static void prod_variant(const pairctx* P, const kspace* s, int n, int kf, int fraglen,
                         float* best, float* gbest, float* tb) {
    refine_loop(P, s, n, kf, fraglen, P->d0fin, P->d0fin * P->d0fin, 0, P->d82, -1.0f, best, tb);
    if (*best < 0.f) { *gbest = *best; return; }   /* nothing computed */
    if (P->lq != P->lr) {
        int gl = P->lq > P->lr ? P->lq : P->lr;
        float g0 = c_d0fin_t(gl, gl, P->rmol);
        *gbest = score_pass(P, s, n, tb, g0 * g0, 0, P->d82, 0, NULL);
    } else *gbest = *best;
}

static void prod_write(pairctx* P, const prodwin* w) {
    float bs = w->best, gb = w->gbest;
    if ((float)P->lr < (float)P->lq) { float t = bs; bs = gb; gb = t; }
    P->out[GTO_SCOREQ] = bs / (float)P->lq;
    P->out[GTO_SCORER] = gb / (float)P->lr;
    P->out[GTO_D0Q] = c_d0fin_t(P->lq, P->lq, P->rmol);
    P->out[GTO_D0R] = c_d0fin_t(P->lr, P->lr, P->rmol);
    memcpy(P->tfm_gr, w->tfm, sizeof(w->tfm));
}

static double rmsd_from_sums(const double* v, double n) {
    /* v: [0..8] sum q_i r_j, [9..11] sum q, [12..14] sum r, [15..17] sum q^2, [18..20] sum r^2 */
    double mq[3], mr[3], S[3][3], E0 = 0.0;
    for (int i = 0; i < 3; i++) { mq[i] = v[9 + i] / n; mr[i] = v[12 + i] / n; }
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) S[i][j] = v[3 * i + j] - n * mq[i] * mr[j];
    for (int i = 0; i < 3; i++) E0 += (v[15 + i] - n * mq[i] * mq[i]) + (v[18 + i] - n * mr[i] * mr[i]);
    double N[4][4];
    double lam = qcp_lambda(S, N);
    double e = (E0 - 2.0 * lam) / n;
    return e > 0.0 ? sqrt(e) : 0.0;
}

/* Production phase 2 by log search (--refinement 0,
 * covariance_production_dp_refn_complete.cu:752-915): from the phase-1
 * position, steps of +-32, 16, ..., 1 positions; at each step the five
 * fragment lengths 1..5 run in order, each carrying the best score so far
 * (the grand best of phase 1 to begin with), and the position moves to the
 * step's position when one of them raised it.  A fragment that reaches past
 * the alignment's end by less than the step is shifted back to end there. */
static void production_logsearch(pairctx* P, const kspace* s, int n) {
    float bestorg = P->grand, best = bestorg, tb[12];
    int posorg = P->sfpos;
    for (int st = 32; st >= 1; st >>= 1)
        for (int sgn = 1; sgn >= -1; sgn -= 2) {
            int step = sgn * st;
            int sfragpos = posorg + step;
            int ext = step > 0 ? step : 0;
            for (int sfragndx = 1; sfragndx < FRAG_NSUB; sfragndx++) {
                int fraglen = frag_length(n, sfragndx);
                if (fraglen < 1) continue;
                if (sfragpos < 0 || n + ext <= sfragpos + fraglen) continue;
                int delta = sfragpos + fraglen - n;
                int kf = sfragpos - (delta > 0 ? delta : 0);
                float bp = best;
                refine_loop(P, s, n, kf, fraglen, P->d0fin, P->d0fin * P->d0fin, 0, P->d82,
                            best, &best, tb);
                if (bp < best) posorg = sfragpos;
            }
        }
    if (best <= bestorg) return;
    prodwin w;
    w.best = best;
    if (P->lq != P->lr) {
        int gl = P->lq > P->lr ? P->lq : P->lr;
        float g0 = c_d0fin_t(gl, gl, P->rmol);
        w.gbest = score_pass(P, s, n, tb, g0 * g0, 0, P->d82, 0, NULL);
    } else w.gbest = best;
    memcpy(w.tfm, tb, sizeof(tb));
    prod_write(P, &w);
}

static void production(pairctx* P, int refinement) {
    kspace s = {1, 0, 0, P->aq, P->ar};
    int n = P->naln;
    int nloc = nlocsteps_refine(P);
    /* phase 1 */
    prodwin w; w.best = 0.f; w.si = -1;
    float rmsd32 = -1.f;
    for (int si = 0; si < nloc && n > 0; si++) {
        int sfragfct = si / FRAG_NSUB, sfragndx = si % FRAG_NSUB;
        int fraglen = frag_length(n, sfragndx);
        if (fraglen < 1) continue;
        int sfragpos = sfragfct * FRAG_STEP;
        if (n + FRAG_STEP <= sfragpos + fraglen) continue;
        int delta = sfragpos + fraglen - n;
        int kf = sfragpos - (delta > 0 ? delta : 0);
        if (si == 0) {
            /* RMSD over the full alignment from compensated FP32 sums */
            float sq[6] = {0}, cq[6] = {0}, bq[6] = {0};
            ccacc a; cc_init(&a);
            int blk = 0;
            for (int k = kf; k < kf + fraglen; k++) {
                int q = P->aq[k], r = P->ar[k];
                float qx = P->qx[q], qy = P->qy[q], qz = P->qz[q];
                float rx = P->rx[r], ry = P->ry[r], rz = P->rz[r];
                cc_add(&a, qx, qy, qz, rx, ry, rz);
                bq[0] = fmaf(qx, qx, bq[0]); bq[1] = fmaf(qy, qy, bq[1]); bq[2] = fmaf(qz, qz, bq[2]);
                bq[3] = fmaf(rx, rx, bq[3]); bq[4] = fmaf(ry, ry, bq[4]); bq[5] = fmaf(rz, rz, bq[5]);
                if (++blk == GTB_BLK) {
                    cc_fold(&a);
                    for (int f = 0; f < 6; f++) nfold(&sq[f], &cq[f], &bq[f]);
                    blk = 0;
                }
            }
            float v[16];
            cc_final(&a, v);
            double dv[21];
            for (int f = 0; f < 15; f++) dv[f] = v[f];
            for (int f = 0; f < 6; f++) { nfold(&sq[f], &cq[f], &bq[f]); dv[15 + f] = (double)(sq[f] + cq[f]); }
            rmsd32 = (float)rmsd_from_sums(dv, (double)fraglen);
        }
        float best, gbest, tb[12];
        prod_variant(P, &s, n, kf, fraglen, &best, &gbest, tb);
        if (best > 0.f && w.best < best) {
            w.best = best; w.gbest = gbest; w.si = si; memcpy(w.tfm, tb, sizeof(tb));
            w.ndx = sfragndx; w.pos = sfragpos;
        }
    }
    if (w.si >= 0) {
        P->grand = w.best;   /* unconditional production save */
        prod_write(P, &w);
        P->sfndx = w.ndx; P->sfpos = w.pos;
    }
    /* phase 2 */
    if (refinement == REF_LOG) production_logsearch(P, &s, n);
    else {
        /* one fragment length (coarse, one-search: MpStageFin.cpp:1310-1525)
         * or every length (full, fullA: covariance_production_dp_refn_complete.cu:381-530,
         * custage_fin.cu:475-481), nf positions around the phase-1 position */
        int full = refinement >= REF_FULL;
        int maxalnmax = P->qmax < P->rmax ? P->qmax : P->rmax;
        int nf = 2 * maxalnmax < FIN_MAXNPOS ? 2 * maxalnmax : FIN_MAXNPOS;
        int nsi = full ? nf * FRAG_NSUB : nf;
        prodwin w2; w2.best = 0.f; w2.si = -1;
        for (int si = 0; si < nsi && n > 0; si++) {
            int sfragfct = full ? si / FRAG_NSUB : si;
            int sfragndx = full ? si % FRAG_NSUB : P->sfndx, sfragpos = P->sfpos;
            sfragpos += (sfragfct - (nf >> 1));
            if (!full && sfragndx == 0) sfragndx++;
            int fraglen = frag_length(n, sfragndx);
            if (fraglen < 1) continue;
            if (sfragpos < 0 || n + 1 <= sfragpos + fraglen) continue;
            float best, gbest, tb[12];
            prod_variant(P, &s, n, sfragpos, fraglen, &best, &gbest, tb);
            if (best > 0.f && w2.best < best) {
                w2.best = best; w2.gbest = gbest; w2.si = si; memcpy(w2.tfm, tb, sizeof(tb));
            }
        }
        if (w2.si >= 0 && P->grand < w2.best) {
            P->grand = w2.best;
            prod_write(P, &w2);
        }
    }
    /* FP64 recomputation of reported values; with --2tm-score also the
     * secondary TM-scores: the same sums without the aligned pairs where one
     * residue is in a helix and the other is not (MpStageFin.cpp:1723-1818,
     * MpStageBase.h:825-856) */
    if (n > 0) {
        double d0q = c_d0fin_t(P->lq, P->lq, P->rmol), d0r = c_d0fin_t(P->lr, P->lr, P->rmol);
        double d0q2 = d0q * d0q, d0r2 = d0r * d0r, tq = 0.0, tr = 0.0, t2q = 0.0, t2r = 0.0;
        double dv[21];
        memset(dv, 0, sizeof(dv));
        const float* t = P->tfm_gr;
        for (int k = 0; k < n; k++) {
            int q = P->aq[k], r = P->ar[k];
            double qx = P->qx[q], qy = P->qy[q], qz = P->qz[q];
            double rx = P->rx[r], ry = P->ry[r], rz = P->rz[r];
            double x = t[0] * qx + t[1] * qy + t[2] * qz + t[9];
            double y = t[3] * qx + t[4] * qy + t[5] * qz + t[10];
            double z = t[6] * qx + t[7] * qy + t[8] * qz + t[11];
            double d = (x - rx) * (x - rx) + (y - ry) * (y - ry) + (z - rz) * (z - rz);
            double sq_ = d0q2 / (d0q2 + d), sr_ = d0r2 / (d0r2 + d);
            tq += sq_;
            tr += sr_;
            char qs = P->qs[q], rs = P->rs[r];
            if (!((qs == 'h' || rs == 'h') && qs != rs)) { t2q += sq_; t2r += sr_; }
            double qq[3] = {qx, qy, qz}, rr[3] = {rx, ry, rz};
            for (int i = 0; i < 3; i++)
                for (int j = 0; j < 3; j++) dv[3 * i + j] += qq[i] * rr[j];
            for (int i = 0; i < 3; i++) {
                dv[9 + i] += qq[i]; dv[12 + i] += rr[i];
                dv[15 + i] += qq[i] * qq[i]; dv[18 + i] += rr[i] * rr[i];
            }
        }
        double r64 = rmsd_from_sums(dv, (double)n);
        if (rmsd32 >= 0.f) {
            P->err[GTO_ERR_RMSD] = (float)fabs((double)rmsd32 - r64);
            P->out[GTO_RMSD] = (float)r64;
        }
        if (P->out[GTO_SCOREQ] > 0.f || P->out[GTO_SCORER] > 0.f) {
            double tmq = tq / P->lq, tmr = tr / P->lr;
            P->err[GTO_ERR_TMQ] = (float)fabs((double)P->out[GTO_SCOREQ] - tmq);
            P->err[GTO_ERR_TMR] = (float)fabs((double)P->out[GTO_SCORER] - tmr);
            P->out[GTO_SCOREQ] = (float)tmq;
            P->out[GTO_SCORER] = (float)tmr;
        }
        if (P->o->twotmscore) {
            P->out[GTO_2SCOREQ] = (float)(t2q / P->lq);
            P->out[GTO_2SCORER] = (float)(t2r / P->lr);
        }
    }
}

/* alignment strings: MpDPHub.cpp:1919-2125 */
static void production_alignment(pairctx* P, char* dst) {
    int W = P->lq + P->lr + 1;
    char *rq = dst, *rm = dst + W, *rt = dst + 2 * W, *sq = dst + 3 * W, *st = dst + 4 * W;
    int n = P->naln, col = 0, psts = 0, idts = 0, gaps = 0;
    unsigned int bc = 0, ec = 0;
    const float d2eq = 25.0f;
    for (int k = 0; k < n; k++) {
        int q = P->aq[k], r = P->ar[k];
        float d = P->ad[k];
        unsigned int cc = ((unsigned int)(r + 1) << 16) | (unsigned int)(q + 1);
        if (k == 0) bc = cc;
        ec = cc;
        int eq = d < d2eq;
        if (eq) psts++;
        char a = (char)P->qa[q], b = (char)P->ra[r];
        rq[col] = a; rt[col] = b; sq[col] = P->qs[q]; st[col] = P->rs[r];
        char mc = eq ? '+' : ' ';
        if (a != '-' && a == b) { idts++; mc = eq ? a : (char)(a | 32); }
        rm[col] = mc;
        col++;
        if (k + 1 < n) {
            int q1 = P->aq[k + 1], r1 = P->ar[k + 1];
            for (int qq = q + 1; qq < q1; qq++) {
                rq[col] = (char)P->qa[qq]; sq[col] = P->qs[qq];
                rt[col] = '-'; st[col] = ' '; rm[col] = ' ';
                col++; gaps++;
            }
            if (!P->o->nodeletions)
                for (int rr = r + 1; rr < r1; rr++) {
                    rt[col] = (char)P->ra[rr]; st[col] = P->rs[rr];
                    rq[col] = '-'; sq[col] = ' '; rm[col] = ' ';
                    col++; gaps++;
                }
        }
    }
    rq[col] = rm[col] = rt[col] = sq[col] = st[col] = 0;
    union { unsigned int u; float f; } ub, ue;
    ub.u = bc; ue.u = ec;
    P->out[GTO_BEGCOORDS] = ub.f;
    P->out[GTO_ENDCOORDS] = ue.f;
    P->out[GTO_ALNLENGTH] = (float)col;
    P->out[GTO_PSTVS] = (float)psts;
    P->out[GTO_IDNTS] = (float)idts;
    P->out[GTO_NGAPS] = (float)gaps;
}

/* ------------------------------------------------------------------------ */
static void run_pair(pairctx* P, char* alndst) {
    const gto_opts* o = P->o;
    /* preinit: MpStage1.cpp:28-167 */
    /* with --pre-similarity active every pair starts filtered, with no
     * molecule-type check, and the ones that pass are released
     * (custage1.cu:74-82, MpStage1.cpp:123-128) */
    int presim = 0.0f < o->presimilarity && PRESIM_EDGE < P->qmax && PRESIM_EDGE < P->rmax;
    if (o->clsfilter) {
        /* a clustering run: every pair starts filtered (CuBatch.cu:452-467) and
         * is released when the reference's global index precedes the end of
         * the query block's and the shorter length reaches the coverage of the
         * longer (coverage.cu:43-51); the screen below only sees the pairs
         * left filtered (similarity.cu:56-65) */
        float lq = (float)P->lq, lr = (float)P->lr;
        float mx = lq < lr ? lr : lq, mn = lq < lr ? lq : lr;
        int pass = o->clsrtype[P->ri] < o->clsqend && mx * o->clscoverage <= mn;
        P->flags = pass ? 0 : CONV_LOWTMSC;
    } else
        P->flags = (presim || P->qmol != P->rmol) ? CONV_LOWTMSC : 0;
    if (presim && P->flags && presim_pass(P, o->presimilarity)) P->flags = 0;
    P->grand = P->best = P->best0 = 0.f;
    P->seedq = P->seedr = 0;
    P->naln = 0;
    P->sfndx = P->sfpos = P->sfndx_cur = P->sfpos_cur = 0;
    tfm_identity(P->tfm_ib);
    tfm_identity(P->tfm_gr);
    memset(P->out, 0, sizeof(P->out));
    memset(P->err, 0, sizeof(P->err));
    P->out[GTO_RMSD] = 9999.9f;
    gto_constants(P->lq, P->lr, &P->d0, &P->d02, &P->d82, &P->d0fin, NULL);
    if (P->rmol) P->d0fin = c_d0fin_na(P->lq, P->lr);
    P->d0s = c_d0s(P->d0);
    float d02dpscan = (P->d0 + 1.5f) * (P->d0 + 1.5f);
    if (alndst) alndst[0] = alndst[P->lq + P->lr + 1] = alndst[2 * (P->lq + P->lr + 1)] =
        alndst[3 * (P->lq + P->lr + 1)] = alndst[4 * (P->lq + P->lr + 1)] = 0;

    /* stage 1 */
    stage1_findfrag(P);
    if (!(P->flags & CONV_LOWTMSC))
        refine_stage(P, 0, P->d0, P->d02, 1, 0.f, 1, 0);
    else P->best = 0.f;
    dprefine(P, 1, 1, 2);

    /* --add-search-by-ss: MpStageSSRR.h:63-76, custage_ssrr.cu:43-140 --
     * the alignment of the DP above, fragment refinement over it, then DP
     * refinement with the gap cost and without, 2 iterations each */
    if (o->addsearchbyss) {
        if (!(P->flags & CONV_LOWTMSC)) {
            dp_ss_run(P, -1.0f);
            btck_matched(P);
        } else P->naln = 0;
        if (P->flags) P->best = 0.f;
        else refine_stage(P, 1, P->d0, P->d02, 1, 0.f, 1, 0);
        dprefine(P, 0, 0, 2);
        dprefine(P, 1, 0, 2);
    }

    /* the spatial-index detailed search (MpBatch.cpp:446-461) */
    if (!o->nodetailedsearch && !(P->flags & CONV_LOWTMSC)) frg3_stage(P);

    /* stage 2, first call: MpStage2.h:63-83 with <false,true,DPSCAN> */
    for (int call = 0; call < 2; call++) {
        int gap0 = call == 1;
        if (!(P->flags & CONV_LOWTMSC)) {
            dp_run(P, P->tfm_gr, gap0, gap0 ? 0.0f : -1.0f, !gap0, gap0 ? P->d02 : d02dpscan);
            if (!(P->flags & CONV_SCOREDP)) btck_matched(P);
            else P->naln = 0;
        } else P->naln = 0;
        if (P->flags) P->best = 0.f;
        else refine_stage(P, 1, P->d0, P->d02, 1, 0.f, 1, 0);
        dprefine(P, 0, 0, 2);
        dprefine(P, 1, 0, call == 0 ? 2 : o->convergence);
        if (call == 1 && 0.0f < o->scorethld) {
            int ml = P->lq < P->lr ? P->lq : P->lr;
            if (P->grand < o->scorethld * (float)ml) P->flags |= CONV_LOWTMSC;
        }
    }

    /* final stage: MpStageFin.h:63-96 */
    if (P->flags & CONV_LOWTMSC) return;
    dp_run(P, P->tfm_gr, 1, 0.f, 0, P->d02);
    btck_matched(P);
    refine_stage(P, 2, P->d0, P->d02, 1, -1.0f, 1, 1);
    if (!(o->depth == 3 || o->refinement == REF_COARSE))
        final_phase2(P, o->refinement == REF_FULLA);
    dp_run(P, P->tfm_gr, 1, 0.f, 0, P->d02);
    btck_constrained(P);
    if (alndst) production_alignment(P, alndst);
    production(P, o->refinement);
    if (o->referenced) {
        float* t = P->tfm_gr;
        float R[9];
        memcpy(R, t, sizeof(R));
        for (int i = 0; i < 3; i++)
            for (int j = 0; j < 3; j++) t[3 * i + j] = R[3 * j + i];
        float t0 = t[9], t1 = t[10], t2 = t[11];
        t[9] = -(R[0] * t0 + R[3] * t1 + R[6] * t2);
        t[10] = -(R[1] * t0 + R[4] * t1 + R[7] * t2);
        t[11] = -(R[2] * t0 + R[5] * t1 + R[8] * t2);
    }
}

int gto_process_block(const gto_opts* o,
                      int nq, const int* qlen, const float* qx, const float* qy,
                      const float* qz, const unsigned char* qrsd, const int* qmol,
                      int nr, const int* rlen, const float* rx, const float* ry,
                      const float* rz, const unsigned char* rrsd, const int* rmol,
                      float* out, float* tfm, float* err,
                      char* alns, const long long* aln_off,
                      char* qss, char* rss, int nthreads) {
    if (!o->nodetailedsearch) return 2;
    return gto_process_block_ndx(o, nq, qlen, qx, qy, qz, qrsd, qmol, NULL, NULL,
                                 nr, rlen, rx, ry, rz, rrsd, rmol, NULL, NULL,
                                 out, tfm, err, alns, aln_off, qss, rss, nthreads);
}

int gto_process_block_ndx(const gto_opts* o,
                          int nq, const int* qlen, const float* qx, const float* qy,
                          const float* qz, const unsigned char* qrsd, const int* qmol,
                          const float* const* qnf, const int* const* qni,
                          int nr, const int* rlen, const float* rx, const float* ry,
                          const float* rz, const unsigned char* rrsd, const int* rmol,
                          const float* const* rnf, const int* const* rni,
                          float* out, float* tfm, float* err,
                          char* alns, const long long* aln_off,
                          char* qss, char* rss, int nthreads) {
    if (nq < 1 || nr < 1) return 1;
    if (!o->nodetailedsearch && (!qnf || !qni || !rnf || !rni)) return 2;
    gtb_gonnet_scores(g_gonnet);
    long long* qoff = (long long*)malloc(sizeof(long long) * (nq + 1));
    long long* roff = (long long*)malloc(sizeof(long long) * (nr + 1));
    qoff[0] = roff[0] = 0;
    int qmax = 0, qmin = 1 << 30, rmax = 0, rmin = 1 << 30;
    for (int i = 0; i < nq; i++) {
        qoff[i + 1] = qoff[i] + qlen[i];
        if (qlen[i] > qmax) qmax = qlen[i];
        if (qlen[i] < qmin) qmin = qlen[i];
    }
    for (int i = 0; i < nr; i++) {
        roff[i + 1] = roff[i] + rlen[i];
        if (rlen[i] > rmax) rmax = rlen[i];
        if (rlen[i] < rmin) rmin = rlen[i];
    }
    /* secondary structure: protein, or nucleic-acid base pairs */
    for (int i = 0; i < nq; i++) {
        long long b = qoff[i];
        if (!qmol || qmol[i] == 0) gto_secstr(qlen[i], qx + b, qy + b, qz + b, qss + b);
        else gto_secstr_na(qlen[i], qx + b, qy + b, qz + b, qrsd + b, qss + b);
    }
    for (int i = 0; i < nr; i++) {
        long long b = roff[i];
        if (!rmol || rmol[i] == 0) gto_secstr(rlen[i], rx + b, ry + b, rz + b, rss + b);
        else gto_secstr_na(rlen[i], rx + b, ry + b, rz + b, rrsd + b, rss + b);
    }
    long long npairs = (long long)nq * nr;
    (void)nthreads;
#pragma omp parallel for schedule(dynamic, 1) num_threads(nthreads > 0 ? nthreads : 1)
    for (long long p = 0; p < npairs; p++) {
        int qi = (int)(p / nr), ri = (int)(p % nr);
        pairctx P;
        memset(&P, 0, sizeof(P));
        P.o = o;
        P.lq = qlen[qi]; P.lr = rlen[ri];
        P.qx = qx + qoff[qi]; P.qy = qy + qoff[qi]; P.qz = qz + qoff[qi];
        P.rx = rx + roff[ri]; P.ry = ry + roff[ri]; P.rz = rz + roff[ri];
        P.qa = qrsd + qoff[qi]; P.ra = rrsd + roff[ri];
        P.qs = qss + qoff[qi]; P.rs = rss + roff[ri];
        P.qmol = qmol ? qmol[qi] : 0; P.rmol = rmol ? rmol[ri] : 0;
        P.ri = ri;
        P.qmax = qmax; P.qmin = qmin; P.rmax = rmax; P.rmin = rmin;
        if (!o->nodetailedsearch) {
            long long a = qoff[qi], b = roff[ri];
            P.qnx = qnf[0] + a; P.qny = qnf[1] + a; P.qnz = qnf[2] + a;
            P.qnl = qni[0] + a; P.qnr = qni[1] + a; P.qno = qni[2] + a;
            P.rnx = rnf[0] + b; P.rny = rnf[1] + b; P.rnz = rnf[2] + b;
            P.rnl = rni[0] + b; P.rnr = rni[1] + b; P.rno = rni[2] + b;
        }
        int mx = P.lq > P.lr ? P.lq : P.lr;
        P.aq = (int*)malloc(sizeof(int) * (mx + 1));
        P.ar = (int*)malloc(sizeof(int) * (mx + 1));
        P.ad = (float*)malloc(sizeof(float) * (mx + 1));
        P.bt = (unsigned char*)malloc((size_t)P.lq * P.lr);
        P.h0 = (float*)malloc(sizeof(float) * P.lr);
        P.h1 = (float*)malloc(sizeof(float) * P.lr);
        run_pair(&P, alns ? alns + aln_off[p] : NULL);
        memcpy(out + p * GTO_NOUT, P.out, sizeof(P.out));
        memcpy(tfm + p * 12, P.tfm_gr, 12 * sizeof(float));
        if (err) memcpy(err + p * GTO_NERR, P.err, sizeof(P.err));
        free(P.aq); free(P.ar); free(P.ad); free(P.bt); free(P.h0); free(P.h1);
    }
    free(qoff);
    free(roff);
    return 0;
}
