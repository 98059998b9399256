// gtb_kernels.cuh -- kernel-side data layout and launchers of the search.
#pragma once
#include <cstdint>
#include <vector>
#include <cuda_runtime.h>

namespace gtb {

// DP traceback storage.  The DP sweeps strips of 32*R query rows (R rows
// per lane of a warp; R = 4 for queries of at least DP_R4_MIN residues, 2
// below) along anti-diagonals, lr + 31 steps per strip rounded up to a
// multiple of 16/R; every lane packs the 2-bit directions of its R rows for
// 16/R consecutive steps into one 32-bit word, words of a strip stored
// [step / (16/R)][lane].
// refinement: pairs with at least RL_LONG positions get RLW_CTAS CTAs of 4
// warps; in the launches where few pairs take part, the pairs below that
// with at least RL_LONG_FEW positions get RLW_CTAS_FEW; a long-pair launch
// has at most RLW_GRID CTAs (they walk the long pairs).  When a sub-batch
// has few pairs of a tier, each gets more CTAs (rlw_ctas_for), up to
// RLW_CTAS_MAX: a lone long pair has variants for many more warps.
constexpr int RL_LONG = 1536;
constexpr int RL_LONG_FEW = 384;
constexpr int RL_NBUCKET = 65536 >> 4;   // work-list buckets; rhist[RL_NBUCKET] = list length
constexpr int RLW_CTAS = 16;
constexpr int RLW_CTAS_FEW = 4;
constexpr int RLW_GRID = 1024;
constexpr int RLW_CTAS_MAX = 256;
constexpr int RLW_CTA_WARPS = 4;     // warps of a long-pair CTA (one candidate each)
// a sub-batch with at most this many pairs in the first long-pair tier runs
// them with a variant per warp (its lanes share each pass) instead of a
// variant per lane: too few variants to fill the lanes otherwise
constexpr int RLW_WIDE_MAX = 64;
constexpr int RLW_CAND = 17;         // floats per warp candidate
// CTAs per pair of a long-pair tier with `nlong` possible pairs: `base`, or
// as many as fill RLW_GRID CTAs, at most RLW_CTAS_MAX
inline int rlw_ctas_for(int base, int nlong) {
    int c = nlong > 0 ? RLW_GRID / nlong : RLW_GRID;
    c = c > base ? c : base;
    return c < RLW_CTAS_MAX ? c : RLW_CTAS_MAX;
}

constexpr int DP_R4_MIN = 384;
__host__ __device__ inline int dp_r(int lq) { return lq >= DP_R4_MIN ? 4 : 2; }
// bytes of a pair's detailed-search region: its local score matrix (lq x lr
// bytes), later the slot DPs' row buffers (32 per section, lr floats each,
// which the DP writes for every strip); a multiple of 16
__host__ __device__ inline long long f3_region_bytes(int lq, int lr, int nsec) {
    long long b = (long long)lq * lr;
    if (b < 128LL * nsec * lr) b = 128LL * nsec * lr;
    return (b + 15) & ~15LL;
}
__host__ __device__ inline long long bt_strip_words(int lr, int R) {
    const int spw = 16 / R;
    return (long long)((lr + 31 + spw - 1) / spw) * 32;
}
// pairs whose DP runs as a wavefront over several CTAs (one warp per strip)
__host__ __device__ inline int dp_strips(int lq) { return (lq + 32 * dp_r(lq) - 1) / (32 * dp_r(lq)); }
__host__ __device__ inline bool dp_wave(int lq, int lr) { return dp_strips(lq) >= 12 && lr >= 512; }
__host__ __device__ inline long long bt_words(int lq, int lr) {
    const int R = dp_r(lq);
    return (long long)((lq + 32 * R - 1) / (32 * R)) * bt_strip_words(lr, R);
}

// Block of queries x references (device pointers, SoA).
struct Blk {
    int nq, nr;
    const int *qlen, *rlen;          // lengths
    const int *qoff, *roff;          // first-residue offsets
    const float *qx, *qy, *qz, *rx, *ry, *rz;
    const float4 *q4, *r4;           // the same coordinates as (x, y, z, 0),
    const int *q4off, *r4off;        // first residue of each structure in q4/r4
    const unsigned char *qa, *ra;    // residue letters
    const char *qs, *rs;             // secondary structure
    const int *qmol, *rmol;          // molecule type per structure
    int qmax, qmin, rmax, rmin;      // block-level length extremes
    const float *t_d0, *t_d82, *t_d0fin;  // per-length constants
    int stepinit, refinement, depth, symmetric, nodeletions;
    int twotm;                       // --2tm-score: record fields 13 and 14
    int addss;                       // --add-search-by-ss
    float presim;                    // --pre-similarity threshold when the screen runs, else 0
    // the spatial-index detailed search (f3 = 1: on): the structures' index
    // trees, packed per node (launch_pack_nodes) at the residue offsets of
    // the coordinates, and its options
    int f3, f3nsec;                  // f3nsec: configuration sections (1..F3_NSEC)
    const float4 *qnd, *rnd;
    const int2 *qnc, *rnc;
    int f3trigger, f3nbranches, f3seedrule, f3window;
    float f3gapcost;
    // clustering runs: the prefilter of CheckMaxCoverage (cls = 1): the
    // references' global indices, the end of the query block's, the coverage
    int cls;
    const int* rtype;
    int clsqend;
    float clscov;
};

// detailed search: fragment slots per configuration section, branches per
// section at most, sections at most (--depth 0: 3, 1: 2, else 1)
constexpr int F3_NTOP = 32;
constexpr int F3_NBMAX = 16;
constexpr int F3_NSEC = 3;

// Batch of consecutive pairs p0 .. p0+np-1 of a block (pair = qi*nr + ri).
struct Bat {
    long long p0;
    int np;
    int *flags, *seedq, *seedr, *naln, *sfndx, *sfpos, *sfndx_cur, *sfpos_cur;
    float *grand, *best, *best0, *rmsd32;
    float *tfm_ib, *tfm_gr;          // [np][12]
    float *out, *err;                // [np][16], [np][4]
    const long long *off_bt;  unsigned* bt;   // traceback words per pair
    const long long *off_row; float* row;     // DP row buffer per pair
    const long long *off_aln; unsigned* aln;  // aligned pairs, reverse order
    float* alc;                      // their coordinates, 6 floats each (offset 6*off_aln)
    const long long *off_str; char* str;      // alignment rows (null: not produced)
    // rows of the pairs with an alignment, packed back to back in str: pair i
    // at str + str_off[i] (-1: none), 5 rows of (columns + 1) bytes each, the
    // last byte of a row its NUL; str_cnt: bytes used
    long long* str_off;
    unsigned long long* str_cnt;
    int *rlist, *rhist;              // refinement work list [np], buckets [4097]
    // long pairs of a refinement launch (null: none possible): list, count,
    // per-pair variant counter, per-warp candidates; rl_nlmax = capacity;
    // this launch's threshold and CTAs per long pair.  The second set (the
    // same fields with 2) is a lower tier, pairs from rl_min2 positions with
    // rlw_ctas2 CTAs each, used in the launches after the --pre-score filter
    // (null rl_long2: no second tier in this launch).  The caller's rlw_ctas
    // is the first tier's CTAs per pair (0: RLW_CTAS)
    int rl_nlmax;
    int rl_min, rlw_ctas;
    int *rl_long, *rl_count, *rl_next;
    float* rl_cand;
    int rl_nlmax2, rl_min2, rlw_ctas2;
    int *rl_long2, *rl_count2, *rl_next2;
    float* rl_cand2;
    int plog_round;                  // round of an RM_PLOG launch (0 .. PLOG_ROUNDS-1)
    // host: a second stream for a refinement launch's long pairs, which then
    // run beside its short pairs (fork and join events; null: one stream)
    cudaStream_t st2;
    cudaEvent_t evfork, evjoin;
    // seed work items when some pair's offsets are split over several CTAs
    // (null: one CTA per pair): item -> pair, item -> chunk, chunks per pair,
    // per-pair packed (score, variant) maximum
    int nff;
    const int *ff_pair, *ff_chunk, *ff_nch;
    unsigned long long* ff_key;
    // long pairs whose DP strips run on several CTAs (null: none): CTA items
    // [slot..., strip offset c...], per slot the pair, its CTA count and the
    // offset of its per-strip progress counters; a per-pair mark; an error flag
    int ndw;
    long long dw_nprog;              // progress counters in dw_prog
    const int *dw_item, *dw_pair, *dw_G;
    const long long* dw_soff;
    const unsigned char* dw_mark;
    int *dw_prog, *dw_err;
    long long dw_spin;               // spins a wavefront wait makes before it gives up
    // the first dp_kc pairs of a DP work list (the largest matrices) run as a
    // wavefront over the 4 warps of a CTA each (0: none; needs dw_err)
    int dp_kc;
    int ff_span;                     // seed offsets per CTA of a split pair (0: FF_CHUNK)
    long long* launches;             // host counter of kernel launches
    cudaError_t* lerr;               // host: first failed launch (null: not recorded)
    struct KTimer* kt;               // host: per-family launch timer (null: off)
    // device work counters (null: not counted), WORK_SLOTS slots per kind
    // (WorkKind), summed on the host
    unsigned long long* work;
    // detailed search (null when off): per pair the local score matrix
    // (lq x lr bytes, row major, at off_lsm[i]); the fragment slots' score
    // and transform, 32 per section ([np][f3nsec * 32][13]); their DP scores
    // ([np][f3nsec * 32]); the branches' transforms and validity, f3br =
    // f3nsec * F3_NBMAX per pair ([np][f3br][12], [np][f3br]); the best
    // branch's transform and score; the refinement variants (1..95, three
    // words per pair) the next DP refinement skips
    const long long* off_lsm;
    unsigned char* lsm;
    float *f3slot, *f3dps, *f3alt, *tfm_2nd, *best2;
    unsigned char* f3ok;
    unsigned* vskip_mask;
    int f3br;
    int alt_rci;                     // DP/traceback of branch alt_rci (-1: none)
    const unsigned* vskip;           // refinement variant skips in force (null: none)
};

// position visits of the seed and refinement passes, DP cells, and the DP
// cells of the detailed search's slot scores
enum WorkKind { WK_SEED = 0, WK_REFINE = 1, WK_DPCELL = 2, WK_F3CELL = 3, WK_NKIND = 4 };

// Device time of the launches of each kernel family, from an event pair
// recorded on the launching stream around each launch (host side).  Where
// sub-batches run concurrently on several streams, a launch's interval also
// covers the other streams' work that overlapped it.
enum KernelFamily { KF_SEED = 0, KF_REFINE = 1, KF_DP = 2, KF_FRG3 = 3, KF_N = 4 };
struct KTimer {
    std::vector<cudaEvent_t> ev;     // begin/end pairs, created on first use
    std::vector<int> fam;
    size_t used = 0;
    void begin(int f, cudaStream_t st);
    void end(cudaStream_t st);
    // adds the elapsed times of the recorded pairs to ms[KF_N] (after they
    // completed) and starts over
    cudaError_t collect(float* ms);
    ~KTimer();
};
struct KtScope {                      // begin/end around one launch helper
    KTimer* k; cudaStream_t st;
    KtScope(const Bat& T, int f, cudaStream_t s) : k(T.kt), st(s) { if (k) k->begin(f, st); }
    ~KtScope() { if (k) k->end(st); }
};
constexpr int WORK_SLOTS = 64;       // spread over addresses: fewer atomic collisions
constexpr long long DP_WAVE_SPIN_DEFAULT = 1LL << 24;
constexpr int DP_CTA_PAIRS = 592;    // dp_kc of the library's runs: 4 CTAs per SM
constexpr int DP_CTA_MAXSTRIPS = 512;   // strips of a 65,535-residue query at 4 rows per lane

// DP cell scores (launch_dp's usess): TM term under a transform, + SS, or the
// --add-search-by-ss score (SS + Gonnet, no transform)
enum DpScore { DP_SC_TFM = 0, DP_SC_TFMSS = 1, DP_SC_SSRR = 2 };
// RM_PLOG: one round of the production phase-2 log search (--refinement -1)
enum RefineMode { RM_INIT = 0, RM_DP = 1, RM_FIN1 = 2, RM_FIN2 = 3, RM_PROD1 = 4, RM_PROD2 = 5,
                  RM_PLOG = 6 };
constexpr int PLOG_ROUNDS = 12;   // steps +-32, +-16, ..., +-1
// the transform a DP uses: iteration best, grand best, the detailed search's
// branch T.alt_rci, or its best branch's result
enum DpTfm { DP_TFM_IBEST = 0, DP_TFM_GRAND = 1, DP_TFM_ALT = 2, DP_TFM_2ND = 3 };

void launch_secstr(char* ss, const float* x, const float* y, const float* z,
                   const int* len, const int* off, const int* mol, int nstr,
                   cudaStream_t st, long long* launches);
// (x, y, z, 0) copies of n coordinates, for single 16-byte loads in the passes
void launch_pack4(float4* out, const float* x, const float* y, const float* z, long long n,
                  cudaStream_t st);
// the same per structure into a back-to-back copy: structure i's residues
// [off[i], off[i]+len[i]) go to out[coff[i] ...]
void launch_pack4_structs(float4* out, const float* x, const float* y, const float* z,
                          const int* off, const int* len, const int* coff, int n,
                          cudaStream_t st);
// index tree nodes packed for the walks: nd[k] = (x, y, z, residue | SS << 16),
// nc[k] = (left, right); n positions of a block (ss: the block's secondary
// structure, computed before)
void launch_pack_nodes(float4* nd, int2* nc, const float* x, const float* y, const float* z,
                       const int* l, const int* r, const int* o, const int* off, const int* len,
                       const char* ss, long long n, int nstr, cudaStream_t st);
void launch_init(const Blk& B, const Bat& T, cudaStream_t st);
// the --pre-similarity screen (B.presim > 0): 20 positions kept from the ends
constexpr int PRESIM_EDGE = 20;
void launch_presim(const Blk& B, const Bat& T, cudaStream_t st);
// Seed offsets per CTA (a pair with more is split over several CTAs).
constexpr int FF_CHUNK = 512;
// the seed's offset index range [silo, sihi] of a pair (MpStage1.cpp:299-318)
__host__ __device__ inline void seed_range(int lq, int lr, int qmax, int qmin, int rmax, int rmin,
                                           int step, int& n1, int& silo, int& sihi, int& prv) {
    int minlenmin = qmin < rmin ? qmin : rmin;
    int minalnmin = (minlenmin >> 1) > 5 ? (minlenmin >> 1) : 5;
    n1 = minalnmin - rmax;
    int n2 = qmax - minalnmin;
    int nsteps = (n2 - n1) / step + 1;
    int ml = lq < lr ? lq : lr;
    prv = (ml >> 1) > 5 ? (ml >> 1) : 5;
    // per-pair admissible offsets: prv - lr <= ab <= lq - prv
    int lo = prv - lr - n1;
    silo = lo <= 0 ? 0 : (lo + step - 1) / step;
    int hi = lq - prv - n1;
    sihi = hi < 0 ? -1 : hi / step;
    if (sihi > nsteps - 1) sihi = nsteps - 1;
}
void launch_findfrag(const Blk& B, const Bat& T, cudaStream_t st);
// few: most pairs of the batch are already filtered out (32 lanes per pair)
void launch_refine(int mode, const Blk& B, const Bat& T, cudaStream_t st, bool few);
// skipmode 0: skip LOWTMSC|SCOREDP (plain), 1: skip LOWTMSC only
void launch_dp(const Blk& B, const Bat& T, int tfmsrc, int gap0, float gcost, int usess,
               int dpscan, int skipmode, cudaStream_t st);
void launch_btck(const Blk& B, const Bat& T, int constrained, cudaStream_t st);
// CTAs that the wavefront DP may keep resident at once on this device
int dp_wave_capacity();
// per-device kernel attributes (shared-memory carve-outs), once per device
void configure_kernels();
void launch_post(const Blk& B, const Bat& T, int dpi, int maxit, int prescreen,
                 float prescore, cudaStream_t st);
void launch_lowscore(const Blk& B, const Bat& T, float thr, cudaStream_t st);
void launch_alnstr(const Blk& B, const Bat& T, cudaStream_t st);
void launch_final(const Blk& B, const Bat& T, int referenced, cudaStream_t st);
// adjoint polishing of the final transforms (steps > 0), before launch_final
void launch_polish_final(const Blk& B, const Bat& T, int steps, cudaStream_t st);
// detailed search (gtb_frg3.cu): the stage between stage 1 and stage 2
void launch_frg3(const Blk& B, const Bat& T, cudaStream_t st);
// work list of the pairs without any flag in skipmask, largest matrices
// first, in T.rlist / T.rhist[RL_NB]
void launch_pair_list(const Blk& B, const Bat& T, int skipmask, cudaStream_t st);
// DP scores (last cell of a gap-0 DP, no traceback) of every pair's 32
// fragment slots with a positive score, over the pair list
void launch_f3_dpscore(const Blk& B, const Bat& T, cudaStream_t st);
void launch_dprefine(const Blk& B, const Bat& T, int gap0, int prescreen, int maxit,
                     float prescore, bool few, int tfm1, cudaStream_t st);
void launch_stages(const Blk& B, const Bat& T, int refinement, int depth, int convergence,
                   float prescore, int referenced, float scorethld, cudaStream_t st,
                   cudaEvent_t* ev, int polish_steps = 0);
// the reader's index trees of n structures (host, gtb_index.cpp)
bool build_index_host(long long n, const int* len, const unsigned* dist, const float* X,
                      const float* Y, const float* Z, long long npos, float* ox, float* oy,
                      float* oz, int* ol, int* orr, int* oo);
// Per-length constant tables (stagecnsts.cuh:48-175), n entries each.
void make_tables(float* d0, float* d82, float* d0fin, int n);

}  // namespace gtb
