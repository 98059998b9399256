/*
 * gtb_gonnet.h -- residue exchange scores of the --add-search-by-ss stage.
 *
 * The published Gonnet, Cohen & Benner (1992) log-odds matrix in tenths
 * (lower triangle, residue order ARNDCQEGHILKMFPSTWYV).  The reference scores
 * a residue pair by log2 of the frequency ratio 10^(G/10), the ratio rounded
 * to 6 decimals (alpha.cpp:167-206), and gives 0 to letters outside the 20
 * amino acids (ratio 1) and to characters outside A..Z (alpha.h:55-60).
 * gtb_gonnet_scores builds that table over the letters A..Z, [a][b] at
 * a * 26 + b, on the host; the device gets the finished table.
 *
 * Plain C: used by the CUDA library's host code and by the CPU oracle.
 */
#ifndef GTB_GONNET_H
#define GTB_GONNET_H

#include <math.h>

#define GTB_GONNET_NA 26

static const char GTB_GONNET_ORDER[21] = "ARNDCQEGHILKMFPSTWYV";

/* row i holds columns 0..i */
static const short GTB_GONNET_TENTHS[210] = {
     24,
     -6,  47,
     -3,   3,  38,
     -3,  -3,  22,  47,
      5, -22, -18, -32, 115,
     -2,  15,   7,   9, -24,  27,
      0,   4,   9,  27, -30,  17,  36,
      5, -10,   4,   1, -20, -10,  -8,  66,
     -8,   6,  12,   4, -13,  12,   4, -14,  60,
     -8, -24, -28, -38, -11, -19, -27, -45, -22,  40,
    -12, -22, -30, -40, -15, -16, -28, -44, -19,  28,  40,
     -4,  27,   8,   5, -28,  15,  12, -11,   6, -21, -21,  32,
     -7, -17, -22, -30,  -9, -10, -20, -35, -13,  25,  28, -14,  43,
    -23, -32, -31, -45,  -8, -26, -39, -52,  -1,  10,  20, -33,  16,  70,
      3,  -9,  -9,  -7, -31,  -2,  -5, -16, -11, -26, -23,  -6, -24, -38,  76,
     11,  -2,   9,   5,   1,   2,   2,   4,  -2, -18, -21,   1, -14, -28,   4,  22,
      6,  -2,   5,   0,  -5,   0,  -1, -11,  -3,  -6, -13,   1,  -6, -22,   1,  15,  25,
    -36, -16, -36, -52, -10, -27, -43, -40,  -8, -18,  -7, -35, -10,  36, -50, -33, -35, 142,
    -22, -18, -14, -28,  -5, -17, -27, -40,  22,  -7,   0, -21,  -2,  51, -31, -19, -19,  41,  78,
      1, -20, -22, -29,   0, -15, -19, -33, -20,  31,  18, -17,  16,   1, -18, -10,   0, -26, -11,  34,
};

static inline int gtb_gonnet_index(char c) {
    for (int k = 0; k < 20; k++)
        if (GTB_GONNET_ORDER[k] == c) return k;
    return -1;
}

/* out[a * 26 + b] = log2(ratio(a, b)) as FP32: logf(ratio) * (float)(1/ln 2) */
static inline void gtb_gonnet_scores(float* out) {
    for (int a = 0; a < GTB_GONNET_NA; a++)
        for (int b = 0; b < GTB_GONNET_NA; b++) {
            int i = gtb_gonnet_index((char)('A' + a)), j = gtb_gonnet_index((char)('A' + b));
            float ratio = 1.0f;
            if (i >= 0 && j >= 0) {
                int g = i >= j ? GTB_GONNET_TENTHS[i * (i + 1) / 2 + j]
                               : GTB_GONNET_TENTHS[j * (j + 1) / 2 + i];
                ratio = (float)(round(pow(10.0, g / 100.0) * 1e6) / 1e6);
            }
            out[a * GTB_GONNET_NA + b] = logf(ratio) * 1.44269504088896338700f;
        }
}

#endif /* GTB_GONNET_H */
