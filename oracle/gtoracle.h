/*
 * gtoracle.h -- CPU oracle for the GTalign per-pair superposition search.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a sequential plain-C restatement of the
 * reference's CPU path (libmymp: MpStage1, MpStageFrg3, MpStage2, MpStageFin,
 * MpDPHub, MpSecStr) used by tests/, __graft_entry__.smoke() and bench.py's
 * cpu_baseline leg as the checker.  The product (gtalign_alpha_b200 and its
 * CUDA library) never links, loads or calls it.
 *
 * Numeric conventions shared with the CUDA path (so results can be compared
 * bit for bit): FP32 coordinates and scores; explicit fused multiply-adds at
 * fixed places and no other contraction; block-compensated (Neumaier) FP32
 * sums in forward position order; FP64 quaternion (QCP) rotation solve; FP64
 * recomputation of the reported TM-scores and RMSD.
 */
#ifndef GTORACLE_H
#define GTORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* per-pair output record; field meaning follows gproc.h TDP2OutputAlnData
 * (src/libgenp/gproc/gproc.h:148-168) */
enum {
    GTO_ORGSTRNO = 0, GTO_STRNEWDST, GTO_BEGCOORDS, GTO_ENDCOORDS,
    GTO_ALNLENGTH, GTO_PSTVS, GTO_IDNTS, GTO_NGAPS, GTO_RMSD,
    GTO_SCOREQ, GTO_SCORER, GTO_D0Q, GTO_D0R, GTO_2SCOREQ, GTO_2SCORER,
    GTO_NOUT = 16
};
/* per-pair numeric-error record: |FP32 path - FP64 recomputation| */
enum { GTO_ERR_TMQ = 0, GTO_ERR_TMR, GTO_ERR_RMSD, GTO_NERR = 4 };

typedef struct {
    int   stepinit;      /* 1 (default depth) or 5 (--depth=3 shallow) */
    int   refinement;    /* the reference's stored code (command line code + 1):
                            0 log search, 1 coarse, 2 one search, 3 full
                            search, 4 full search in both final phases */
    int   depth;         /* 0..3 (3 = shallow) */
    int   convergence;   /* --convergence (max DP iterations in stage 2b) */
    float prescore;      /* --pre-score */
    float scorethld;     /* -s */
    int   symmetric;     /* --symmetric */
    int   referenced;    /* --referenced */
    int   nodeletions;   /* --no-deletions */
    int   twotmscore;    /* --2tm-score */
    int   addsearchbyss; /* --add-search-by-ss */
    float presimilarity; /* --pre-similarity (0: off) */
    /* the spatial-index detailed search (MpStageFrg3) */
    int   nodetailedsearch; /* --no-detailed-search */
    int   trigger;       /* --trigger 0..100 (percent) */
    int   nbranches;     /* --nbranches */
    float gapcost;       /* --gapcost as the cost: -0.8, -1.2 or -3.0 */
    int   seedrule;      /* --seedrule as the frame: 0, 64 or 128 */
    int   window;        /* --window 256..512 */
    /* a clustering run's prefilter (CheckMaxCoverage, cufilter/coverage.cu:28-52):
     * the references' global indices (pps2DType), the end of the query
     * block's (qrysernrbeg + nqystrs), --cls-coverage */
    int   clsfilter;
    const int* clsrtype;
    int   clsqend;
    float clscoverage;
} gto_opts;

/* Process a block of nq queries x nr references.
 * Coordinates are SoA, structures concatenated (offsets = prefix sums of
 * lengths).  rsd: residue letters.  mol: molecule type (0 protein, 1 NA).
 * out: [nq*nr][GTO_NOUT]; tfm: [nq*nr][12]; err: [nq*nr][GTO_NERR] (may be
 * NULL); alns: [nq*nr] pointers? -- no: alns is one buffer, pair p owns
 * 5*(lq+lr+1) bytes at aln_off[p] (rows query, middle, target, query SS,
 * target SS, each lq+lr+1 long, NUL-terminated).
 * qss/rss: secondary structure outputs (length = total residues).
 * Returns 0 on success. */
int gto_process_block(const gto_opts* o,
                      int nq, const int* qlen, const float* qx, const float* qy,
                      const float* qz, const unsigned char* qrsd, const int* qmol,
                      int nr, const int* rlen, const float* rx, const float* ry,
                      const float* rz, const unsigned char* rrsd, const int* rmol,
                      float* out, float* tfm, float* err,
                      char* alns, const long long* aln_off,
                      char* qss, char* rss, int nthreads);

/* The same with the blocks' index trees (the reader's six index fields per
 * block, structures concatenated like the coordinates: node coordinates,
 * left and right child, residue), needed when o->nodetailedsearch is 0. */
int gto_process_block_ndx(const gto_opts* o,
                          int nq, const int* qlen, const float* qx, const float* qy,
                          const float* qz, const unsigned char* qrsd, const int* qmol,
                          const float* const* qnf, const int* const* qni,
                          int nr, const int* rlen, const float* rx, const float* ry,
                          const float* rz, const unsigned char* rrsd, const int* rmol,
                          const float* const* rnf, const int* const* rni,
                          float* out, float* tfm, float* err,
                          char* alns, const long long* aln_off,
                          char* qss, char* rss, int nthreads);

/* single building blocks (exposed for unit tests) */
void gto_secstr(int len, const float* x, const float* y, const float* z, char* ss);
void gto_secstr_na(int len, const float* x, const float* y, const float* z,
                   const unsigned char* rsd, char* ss);
int  gto_solve(const float* sums15, int n, float* tfm12);
void gto_constants(int lq, int lr, float* d0, float* d02, float* d82,
                   float* d0fin, float* d02dpscan);

#ifdef __cplusplus
}
#endif
#endif
