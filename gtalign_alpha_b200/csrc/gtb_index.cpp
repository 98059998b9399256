// gtb_index.cpp -- the per-structure 3-d tree index of a block (host code).
//
// The reference's reader builds, next to each SoA batch, six index fields
// (PM2DVectorFields.h:260-281; PMBatchStrDataIndex::MakeIndex,
// src/libgenp/gdats/PMBatchStrDataIndex.cpp) that its spatial-index search
// walks: for every structure, a 3-d tree over its residues stored in the
// structure's own position range, node n at the same offset as a residue:
// the node's coordinates (3 floats), its left and right child nodes (int,
// -1: none) and the residue it holds (int).  The tree of positions
// [b, e) puts the median (b + (e - b)/2, by the coordinate of the level's
// axis x, y, z cycling with depth) at that position and recurses on both
// halves.  The median is chosen by the C++ standard library's selection
// algorithm over the residue indices, as the reader does, so the same input
// gives the same tree node for node (the search below visits a bounded
// number of nodes, so the exact tree matters for its results).
#include <algorithm>
#include <numeric>
#include <vector>
#include <cstring>

#include "gtb200.h"

namespace {

struct Tree {
    const float* c[3];      // the structure's coordinates
    int* left;
    int* right;
    std::vector<int> ndx;   // residue held by each node position
};

int construct(Tree& T, int begin, int end, int dim) {
    if (end <= begin) return -1;
    const int n = begin + ((end - begin) >> 1);
    const float* cd = T.c[dim];
    std::nth_element(T.ndx.begin() + begin, T.ndx.begin() + n, T.ndx.begin() + end,
                     [cd](int a, int b) { return cd[a] < cd[b]; });
    const int nd = (dim + 1) % 3;
    T.left[n] = construct(T, begin, n, nd);
    T.right[n] = construct(T, n + 1, end, nd);
    return n;
}

}  // namespace

namespace gtb {
// The index of n structures (lengths len, first residues dist, coordinates
// X/Y/Z of npos residues) into ox/oy/oz/ol/orr/oo.  Returns false on
// inconsistent input.
bool build_index_host(long long n, const int* len, const unsigned* dist, const float* X,
                      const float* Y, const float* Z, long long npos, float* ox, float* oy,
                      float* oz, int* ol, int* orr, int* oo) {
    for (long long s = 0; s < n; s++) {
        const int L = len[s];
        const long long a = dist[s];
        if (L < 0 || a < 0 || a + L > npos) return false;
        if (L < 1) continue;
        Tree T;
        T.c[0] = X + a; T.c[1] = Y + a; T.c[2] = Z + a;
        T.left = ol + a;
        T.right = orr + a;
        T.ndx.resize(L);
        std::iota(T.ndx.begin(), T.ndx.end(), 0);
        construct(T, 0, L, 0);
        for (int k = 0; k < L; k++) {
            const int r = T.ndx[k];
            ox[a + k] = X[a + r];
            oy[a + k] = Y[a + r];
            oz[a + k] = Z[a + r];
            oo[a + k] = r;
        }
    }
    return true;
}
}  // namespace gtb

extern "C" gtb_status gtb_build_index(char* const* pmbeg, char* const* pmend,
                                      char* const* ndxbeg) {
    if (!pmbeg || !pmend || !ndxbeg) return GTB_ERR_ARG;
    const long long n = (pmend[GTB_FLD_LEN] - pmbeg[GTB_FLD_LEN]) / (long long)sizeof(int);
    if (n < 0) return GTB_ERR_ARG;
    const int* len = (const int*)pmbeg[GTB_FLD_LEN];
    const unsigned* dist = (const unsigned*)pmbeg[GTB_FLD_DIST];
    const float* X = (const float*)pmbeg[GTB_FLD_X];
    const float* Y = (const float*)pmbeg[GTB_FLD_Y];
    const float* Z = (const float*)pmbeg[GTB_FLD_Z];
    float* ox = (float*)ndxbeg[GTB_NDX_X];
    float* oy = (float*)ndxbeg[GTB_NDX_Y];
    float* oz = (float*)ndxbeg[GTB_NDX_Z];
    int* ol = (int*)ndxbeg[GTB_NDX_LEFT];
    int* orr = (int*)ndxbeg[GTB_NDX_RIGHT];
    int* oo = (int*)ndxbeg[GTB_NDX_ORGNDX];
    if (!len || !dist || !X || !Y || !Z || !ox || !oy || !oz || !ol || !orr || !oo) return GTB_ERR_ARG;
    const long long npos = (pmend[GTB_FLD_X] - pmbeg[GTB_FLD_X]) / (long long)sizeof(float);
    return gtb::build_index_host(n, len, dist, X, Y, Z, npos, ox, oy, oz, ol, orr, oo)
               ? GTB_OK : GTB_ERR_ARG;
}
