/*
 * gtb200.h -- C ABI of the B200 (sm_100a) GTalign superposition-search library.
 *
 * Drop-in replacement for the stage sequence beneath CuBatch::ProcessBlock of
 * the reference (src/libmycu/cubatch/CuBatch.cuh:74-85, defined at
 * src/libmycu/cubatch/CuBatch.cu:339-717): the same SoA structure batches in,
 * the same per-pair result records, 12-float transformation matrices and
 * alignment rows out.  Plain C types only; errors are status codes (no C++
 * exceptions cross this boundary).
 *
 * Threading: one handle per host thread / device area, as the reference's
 * CuBatch (one stream per call, CuBatch.cu:420).  A handle is not reentrant.
 */
#ifndef GTB200_H
#define GTB200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    GTB_OK = 0,
    GTB_ERR_ARG = 1,          /* invalid argument (null pointer, bad size) */
    GTB_ERR_CUDA = 2,         /* CUDA runtime error; see gtb_last_error */
    GTB_ERR_NOMEM = 3,        /* the block does not fit the device memory budget */
    GTB_ERR_UNSUPPORTED = 4,  /* option combination not implemented */
    GTB_ERR_TOO_LONG = 5,     /* structure longer than 65535 residues */
    GTB_ERR_NOT_BUILT = 6     /* library built without device code */
} gtb_status;

/* --refinement codes of the gtalign command line (gtalign.h:154-156); the
 * reference stores code + 1 (gtalign.cpp:776-780, CLOptions.h:121-128) */
enum {
    GTB_REFINEMENT_LOG = -1,    /* production phase 2 by log search */
    GTB_REFINEMENT_COARSE = 0,  /* no final phase 2 (the --speed 10..13 presets) */
    GTB_REFINEMENT_ONE = 1,     /* one fragment length in phase 2 (default) */
    GTB_REFINEMENT_FULL = 2,    /* every fragment length in production phase 2 */
    GTB_REFINEMENT_FULLA = 3    /* every fragment length in both final phases 2 */
};

/* Field indices of the reference's SoA batch (PM2DVectorFields.h:220-239):
 * pmbeg[f]/pmend[f] delimit field f over all structures of a block. */
enum {
    GTB_FLD_LEN = 0,      /* int32 structure length (pps2DLen) */
    GTB_FLD_DIST = 1,     /* uint32 offset of the structure's first residue (pps2DDist) */
    GTB_FLD_TYPE = 2,     /* int32 (pps2DType): a clustering run's global
                             structure index, read only when clsfilter is 1 */
    GTB_FLD_X = 3,        /* float x (pmv2DCoords+0) */
    GTB_FLD_Y = 4,        /* float y */
    GTB_FLD_Z = 5,        /* float z */
    GTB_FLD_INSCHORD = 6, /* int32; sign of the first residue's value = molecule type:
                             > 0 nucleic acid, <= 0 protein (GetMoleculeType) */
    GTB_FLD_RESNUM = 7,   /* int32 residue number (unused here) */
    GTB_FLD_RSD = 8,      /* char residue letter (pmv2Drsd) */
    GTB_FLD_SS = 9,       /* char secondary structure (pmv2Dss; computed here) */
    GTB_NFIELDS = 10
};

/* Index fields of a block (PM2DVectorFields.h:260-281): per structure a 3-d
 * tree over its residues in the structure's own position range; node n holds
 * coordinates x, y, z (float), its left and right child nodes (int32, -1 for
 * none) and the residue it stands for (int32).  The reader makes them
 * (PMBatchStrDataIndex::MakeIndex, PMBatchStrDataIndex.cpp); the
 * spatial-index detailed search reads them. */
enum {
    GTB_NDX_X = 0, GTB_NDX_Y = 1, GTB_NDX_Z = 2,
    GTB_NDX_LEFT = 3, GTB_NDX_RIGHT = 4, GTB_NDX_ORGNDX = 5,
    GTB_NNDXFIELDS = 6
};

/* Per-pair output record (gproc.h:148-168, TDP2OutputAlnData) */
enum {
    GTB_OUT_ORGSTRNO = 0, GTB_OUT_STRNEWDST = 1, GTB_OUT_BEGCOORDS = 2,
    GTB_OUT_ENDCOORDS = 3, GTB_OUT_ALNLENGTH = 4, GTB_OUT_PSTVS = 5,
    GTB_OUT_IDNTS = 6, GTB_OUT_NGAPS = 7, GTB_OUT_RMSD = 8, GTB_OUT_SCOREQ = 9,
    GTB_OUT_SCORER = 10, GTB_OUT_D0Q = 11, GTB_OUT_D0R = 12,
    GTB_OUT_2SCOREQ = 13, GTB_OUT_2SCORER = 14, GTB_NOUT = 16
};
/* Per-pair numeric error record: |FP32 search path - FP64 recomputation| */
enum { GTB_ERR_TMQ = 0, GTB_ERR_TMR = 1, GTB_ERR_RMSD = 2, GTB_NERR = 4 };

/* Options the path reads (CuBatch.cu:353-366, custage_fin.cu:243-245,409),
 * with the values of the gtalign command line. */
typedef struct {
    int   refinement;        /* --refinement (GTB_REFINEMENT_*): -1 log search,
                                0 coarse, 1 one search (default), 2 full search,
                                3 full search in both final phases */
    int   depth;             /* --depth 0..3 (3 = shallow: seed step 5) */
    int   convergence;       /* --convergence 1..30 */
    float prescore;          /* --pre-score [0,1) */
    int   symmetric;         /* --symmetric */
    int   referenced;        /* --referenced */
    int   nodeletions;       /* --no-deletions */
    int   nodetailedsearch;  /* --no-detailed-search: 0 runs the spatial-index
                                detailed search (MpStageFrg3) between stage 1
                                and stage 2, as the reference does at --speed
                                <= 12; its options are the last five below */
    int   addsearchbyss;     /* --add-search-by-ss: after stage 1, an alignment
                                by secondary structure and residue similarity,
                                refined like stage 2's */
    int   twotmscore;        /* --2tm-score: record fields GTB_OUT_2SCOREQ/R get
                                the TM-scores without the aligned pairs of a
                                helix and a non-helix residue */
    int   polish_steps;      /* no reference counterpart: 0 (the reference's
                                results) or 1..50 projected-gradient steps on
                                SO(3) x R^3 that polish each pair's final
                                transform with the TM-score adjoint before the
                                FP64 recomputation; a step is kept only if it
                                raises the TM-score (d0 of the shorter
                                structure) over the final alignment */
    float presimilarity;     /* --pre-similarity: 0 (off) or the score an
                                ungapped run of Gonnet residue scores on some
                                diagonal of a pair must reach for the pair to
                                be compared at all */
    /* the detailed search (read when nodetailedsearch is 0), the command
     * line's codes (CLOptions.h:122-160, gtalign.h:157-186) */
    int   trigger;           /* --trigger 0..100 (default 50) */
    int   nbranches;         /* --nbranches 1..16 (default 5) */
    int   gapcost;           /* --gapcost 0..2 (-0.8, -1.2, -3.0; default 1) */
    int   seedrule;          /* --seedrule 0..2 (fragments, 64- or 128-residue
                                local alignment frames; default 1) */
    int   window;            /* --window 256..512 (default 256) */
    /* clustering runs (--cls): every pair starts filtered and is compared
     * only when the reference's global index (GTB_FLD_TYPE, pps2DType) is below
     * the end of the query block's (its smallest + its count: the block's
     * indices are consecutive, TdClustWriter.h:213-219) and the shorter length
     * is at least clscoverage x the longer (CheckMaxCoverage,
     * cufilter/coverage.cu:28-52, CuBatch.cu:452-495) */
    int   clsfilter;         /* 1 in a clustering run */
    float clscoverage;       /* --cls-coverage (default 0.7) */
} gtb_options;

/* Result buffers (host memory), sizes for nq queries x nr references with
 * total residue counts Nq, Nr:
 *   alndata: nq*nr*GTB_NOUT floats    (record of pair (qi,ri) at (qi*nr+ri)*GTB_NOUT)
 *   tfm:     nq*nr*12 floats          (row-major rotation, then translation;
 *                                      transforms the query onto the reference,
 *                                      or the reverse with --referenced)
 *   alns:    sum over qi of 5*(Nr + nr*(lq_i+1)) bytes, the reference's layout
 *            (MpDPHub.cpp:1975-1981): for query qi, 5 rows (query, middle,
 *            target, query SS, target SS) of length Nr + nr*(lq_i+1); pair
 *            (qi,ri) starts at column dist_ri + ri*(lq_i+1); NUL-terminated.
 *            May be NULL.
 *   numerr:  nq*nr*GTB_NERR floats; may be NULL.
 *   qss/rss: Nq / Nr secondary-structure letters; may be NULL. */
typedef struct {
    float* alndata;
    float* tfm;
    char*  alns;
    float* numerr;
    char*  qss;
    char*  rss;
} gtb_results;

typedef struct gtb_handle gtb_handle;

/* Create a handle on CUDA device `device` with a device-memory budget of
 * `mem_bytes` (0 = all free memory minus 256 MB; the --dev-mem analogue,
 * Devices.cu:206-213).  Replaces the construction of CuDeviceMemory + CuBatch. */
gtb_status gtb_create(int device, size_t mem_bytes, const gtb_options* opts,
                      gtb_handle** out);

/* Align every query of a block with every reference of a block.
 * Replaces CuBatch::TransferQueryPMDataToDevice + TransferCPMDataToDevice +
 * CuBatch::ProcessBlock (CuBatch.cuh:54-85).  querypmbeg/querypmend and
 * bdbCpmbeg/bdbCpmend are arrays of GTB_NFIELDS host pointers delimiting each
 * SoA field, exactly as PMBatchStrData hands them to the reference.
 * scorethld is the -s threshold.  All buffers are host memory; the call
 * copies inputs to the device and results back before returning. */
gtb_status gtb_process_block(gtb_handle* h, float scorethld,
                             char* const* querypmbeg, char* const* querypmend,
                             char* const* bdbCpmbeg, char* const* bdbCpmend,
                             gtb_results* out);

/* The same with the blocks' index fields as the reader made them
 * (queryndxpmbeg / bdbCndxpmbeg: GTB_NNDXFIELDS host pointers each, the
 * index data CuBatch transfers beside the SoA fields, CuBatch.cuh:54-72).
 * gtb_process_block builds them itself (gtb_build_index) when the detailed
 * search is on; a reader that has them saves that work. */
gtb_status gtb_process_block_ndx(gtb_handle* h, float scorethld,
                                 char* const* querypmbeg, char* const* querypmend,
                                 char* const* queryndxpmbeg,
                                 char* const* bdbCpmbeg, char* const* bdbCpmend,
                                 char* const* bdbCndxpmbeg, gtb_results* out);

/* Device-resident blocks: the reference uploads a reference chunk once and
 * reuses it for every query block (TdCommutator.cpp:265-285,
 * CuDeviceMemory::TransferCPMDataToDevice); gtb_block_upload is that step.
 * gtb_process_resident aligns two resident blocks and writes the result
 * records, transforms and (optionally) numeric errors to DEVICE buffers of
 * the sizes given for gtb_results (no alignment rows). */
typedef struct gtb_block gtb_block;
gtb_status gtb_block_upload(gtb_handle* h, char* const* pmbeg, char* const* pmend,
                            gtb_block** out);
/* The same with the block's index fields (GTB_NNDXFIELDS host pointers; NULL:
 * built here when the handle's detailed search is on). */
gtb_status gtb_block_upload_ndx(gtb_handle* h, char* const* pmbeg, char* const* pmend,
                                char* const* ndxbeg, gtb_block** out);
/* Free a block with the handle that uploaded it, before gtb_destroy. */
void gtb_block_free(gtb_handle* h, gtb_block* b);
gtb_status gtb_process_resident(gtb_handle* h, float scorethld, const gtb_block* queries,
                                const gtb_block* refs, float* d_alndata, float* d_tfm,
                                float* d_numerr);

/* Build the index fields of a block (replaces PMBatchStrDataIndex::MakeIndex,
 * src/libgenp/gdats/PMBatchStrDataIndex.cpp:48-110, for callers that do not
 * run the reference's reader): ndxbeg[GTB_NNDXFIELDS] are host arrays of as
 * many entries as the block has residues (x, y, z float; left, right, residue
 * int32).  The tree is the reader's, node for node.  Host code. */
gtb_status gtb_build_index(char* const* pmbeg, char* const* pmend, char* const* ndxbeg);

/* Total bytes of the alns buffer for a block (GetSizeOfDP2Alns,
 * CuMemoryBase.h:150-158). */
size_t gtb_alns_size(char* const* querypmbeg, char* const* querypmend,
                     char* const* bdbCpmbeg, char* const* bdbCpmend);

/* Adjoint of the TM-score for fixed alignments (no reference counterpart:
 * the superposition-polishing extension of this library).
 * For npairs pairs, pair p has n_p aligned residue pairs at aln offset
 * off[p] (arrays qxyz/rxyz hold 3*sum(n_p) floats, xyz interleaved per
 * residue), a transform tfm[p*12..] and a d0 value d0[p].  Computes
 * tm[p] = sum_i d0^2/(d0^2 + |R q_i + t - r_i|^2) and its gradient with
 * respect to the rotation vector (omega, a left-multiplied infinitesimal
 * rotation) and the translation: grad[p*6..] = (dTM/domega_xyz, dTM/dt_xyz).
 * When gq is non-NULL the per-residue gradient with respect to the query
 * coordinates is written to gq (3*sum(n_p)).  Device pointers, stream. */
gtb_status gtb_tm_adjoint(gtb_handle* h, int npairs, const long long* off,
                          const int* n, const float* qxyz, const float* rxyz,
                          const float* tfm, const float* d0,
                          float* tm, float* grad, float* gq, void* stream);

/* Projected-gradient polishing of transforms on SO(3) x R^3 for fixed
 * alignments: `steps` ascent steps with backtracking; a step is only
 * accepted when it does not lower the TM-score.  Device pointers, stream.
 * tm_before/tm_after receive the scores (may be NULL). */
gtb_status gtb_polish(gtb_handle* h, int npairs, const long long* off,
                      const int* n, const float* qxyz, const float* rxyz,
                      float* tfm, const float* d0, int steps,
                      float* tm_before, float* tm_after, void* stream);

/* ---------------------------------------------------------------------------
 * Allocation-free search (no counterpart in the reference).
 *
 * For callers that must not allocate device memory while they align
 * structures -- code living inside another framework's memory pool, a
 * process whose device footprint must stay fixed after start-up, or code
 * running while an allocator is locked.  Inputs and outputs are the
 * caller's own device buffers; all working memory comes from one static
 * device array of GTB_NOALLOC_SCRATCH_BYTES (16 MiB) that every GPU loading
 * this library keeps until the process exits.  The call uses no handle and
 * calls no cudaMalloc/cudaFree.  Blocks whose working memory would exceed the
 * array, or with more than GTB_NOALLOC_MAX_PAIRS pairs, are rejected with
 * GTB_ERR_NOMEM and a message in errbuf.  The first call on a device performs
 * a one-time set-up there (device addresses of the static arrays, constant
 * tables): make it before any stream capture.  All calls on one device share
 * that device's scratch array, so calls that overlap on the same GPU race;
 * issue them one after another.  Host threads calling on different devices
 * at once do not conflict.  The caller's current device is restored before
 * the call returns.  Results are those of gtb_process_block (records and
 * transforms only).  Blocks that would pair two nucleic-acid structures are
 * refused with GTB_ERR_UNSUPPORTED, as by gtb_process_block (the molecule
 * types are read back from the device before any search work), and so are
 * options with the detailed search on (nodetailedsearch 0) or a clustering
 * run's prefilter (clsfilter 1): this path carries no index trees and no
 * global indices. */
#define GTB_NOALLOC_SCRATCH_BYTES ((size_t)16 << 20)
#define GTB_NOALLOC_MAX_PAIRS 4096

typedef struct {
    int n;                     /* number of structures */
    const int* lens;           /* HOST copy of the n lengths (working-memory plan) */
    const int* d_lens;         /* device: lengths */
    const int* d_offs;         /* device: offset of each structure's first residue */
    const int* d_mol;          /* device: molecule type (0 protein, 1 nucleic acid) */
    const float *d_x, *d_y, *d_z;
    const unsigned char* d_rsd;  /* device: residue letters */
    char* d_ss;                /* device output: secondary structure per residue */
} gtb_dev_soa;

gtb_status gtb_process_block_noalloc(int device, const gtb_options* opts, float scorethld,
                                     const gtb_dev_soa* queries, const gtb_dev_soa* refs,
                                     float* d_alndata, float* d_tfm, float* d_numerr,
                                     void* stream, char* errbuf, size_t errlen);

/* Message of the last error on this handle (static storage of the handle). */
const char* gtb_last_error(const gtb_handle* h);

/* Number of kernel launches issued by the last gtb_process_block call. */
long long gtb_last_launch_count(const gtb_handle* h);

/* Device time (ms) of the last gtb_process_block call, per stage:
 * [0] stage-1 seed, [1] stage-1 fragment refinement, [2] the DP <->
 * refinement loops (stage-1 DPRefine and both stage-2 passes), [3] and [4]
 * unused (0), [5] final + production stages, [6] total.  A batch runs as up
 * to three concurrent sub-batches; the times are summed over them. */
gtb_status gtb_last_timings(const gtb_handle* h, float* ms7);

/* Algorithmic work of the last gtb_process_block / gtb_process_resident
 * call, counted on the device (no reference counterpart; the measurement
 * behind a FP32 roofline): w4[0] position visits of the seed passes (one
 * visit = one aligned residue pair transformed, scored or added to a
 * covariance in one pass), w4[1] position visits of the refinement passes,
 * w4[2] DP matrix cells, w4[3] DP matrix cells of the detailed search's
 * fragment-slot scores. */
gtb_status gtb_last_work(const gtb_handle* h, unsigned long long* w4);

/* Per-family device time (no reference counterpart): with timing on, every
 * launch of the seed scan, the refinement passes, the DP and the detailed
 * search's own kernels is bracketed by CUDA events on its stream, and
 * gtb_last_kernel_ms gives the summed times (ms) of the last call:
 * ms4[0] seed, [1] refinement, [2] DP, [3] detailed search.  Launches of
 * concurrent sub-batches overlap, so a sum can exceed the call's span.
 * Off by default. */
gtb_status gtb_set_kernel_timing(gtb_handle* h, int on);
gtb_status gtb_last_kernel_ms(const gtb_handle* h, float* ms4);

/* Spins a bounded wait of the wavefront DPs (a long pair's strips over
 * several CTAs, or a large pair's over the warps of one CTA) makes before it
 * gives up (no reference counterpart; default 2^24).  A wait that gives up ends the call
 * with GTB_ERR_CUDA and a message; the handle stays usable.  Small values
 * make the waits give up early, which is how the failure path is tested. */
gtb_status gtb_set_wait_limit(gtb_handle* h, long long spins);

/* Launch shapes of a handle (no reference counterpart: the reference fixes
 * its launch configurations at compile time).  None of them changes a
 * result, only how the work is spread over the SMs and streams. */
typedef struct {
    int seed_chunk;        /* seed offsets per CTA; a pair with more is split
                              over several CTAs (128..65536; default 512) */
    int refine_long_ctas;  /* CTAs per pair of the refinement's long-pair tier
                              (pairs from 1,536 positions; 1..16; default 16);
                              raised, up to 256, where a sub-batch has so few
                              such pairs that their launch would have fewer
                              than 1,024 CTAs */
    int dp_cta_pairs;      /* pairs of each DP launch (its largest matrices)
                              run as a wavefront over a CTA's warps
                              (0..65536; default 592, 4 per SM) */
    int sub_pairs;         /* pairs per concurrent sub-batch, at least
                              (1024..2^30; default 16384) */
} gtb_tuning;
gtb_status gtb_get_tuning(const gtb_handle* h, gtb_tuning* t);
/* GTB_ERR_ARG (the handle's tuning unchanged) when a field is out of range. */
gtb_status gtb_set_tuning(gtb_handle* h, const gtb_tuning* t);

/* Autotuner: times gtb_process_resident on two resident blocks (a sample of
 * the caller's workload, or the workload itself) for candidate launch
 * shapes, one field at a time from the handle's current tuning (seed_chunk
 * 256/512/1024/2048, refine_long_ctas 4/8/16, dp_cta_pairs 0/296/592/1184,
 * sub_pairs 8192/16384/32768); a candidate replaces the field's value only
 * when its time, the least of `trials` calls after one untimed call (two
 * for the starting tuning), is below 98% of the best so far.  Leaves the winner set on the handle and
 * returns it in *best and its time in *best_ms (either may be NULL).
 * `log`, when not NULL, receives up to `nlog` entries (the tuning tried
 * and its ms) and *nlogged their count.  Host wall time around the calls,
 * which synchronise; the results written by the calls are discarded. */
typedef struct {
    gtb_tuning t;
    float ms;
} gtb_tuning_trial;
gtb_status gtb_autotune(gtb_handle* h, float scorethld, const gtb_block* queries,
                        const gtb_block* refs, int trials, gtb_tuning* best, float* best_ms,
                        gtb_tuning_trial* log, int nlog, int* nlogged);

void gtb_destroy(gtb_handle* h);

/* Host reader and packer (replaces, for callers without the reference's
 * reader, FlexDataRead::ReadDataPDB + PMBatchStrData::AddOneResidue /
 * FinalizeCrntStructure, src/libgenp/gdats/FlexDataRead.cpp:285-930,
 * PMBatchStrData.h:368-545): PDB and PDBx/mmCIF files, plain or
 * gzip-compressed, parsed on
 * `nthreads` host threads (0: all cores) into one block of the SoA fields
 * above, structures in file order, as the reference's reader produces them
 * under the same interpretation options; tar archives are read entry by
 * entry (descriptions "<archive>:<entry>").  Host code; needs no device. */
typedef struct {
    int ter;          /* --ter: 0 end of file, 1 ENDMDL/END, 2 + chain change,
                         3 + TER (default 3) */
    int split;        /* --split: 0 none, 1 each MODEL (with ter 0), 2 each chain
                         (with ter 0 or 1) (default 0) */
    int hetatm;       /* --hetatm: HETATM records too (default 0) */
    int mol;          /* --mol: 0 protein, 1 nucleic acid, 2 by residue name (default 2) */
    char aatom[5];    /* --aatom, 4 characters (default " CA ") */
    char natom[5];    /* --natom, 4 characters (default " C3'") */
    int minlen;       /* --dev-min-length: shorter structures are dropped (default 20) */
    int maxlen;       /* --dev-max-length: longer ones are dropped (default 65535;
                         the reference's default for references is 4000) */
    int infmt;        /* --infmt: 0 by the file name (.cif, .cif.gz: PDBx/mmCIF;
                         else PDB), 1 PDB, 2 PDBx/mmCIF (default 0) */
} gtb_reader_options;
typedef struct gtb_structs gtb_structs;
void gtb_reader_default_options(gtb_reader_options* o);
/* err: a message of at most errlen bytes on failure (may be NULL). */
gtb_status gtb_read_pdb(const char* const* paths, int npaths, const gtb_reader_options* opts,
                        int nthreads, gtb_structs** out, char* err, size_t errlen);
gtb_status gtb_structs_size(const gtb_structs* b, int* nstr, long long* npos);
/* The block's GTB_NFIELDS field pointers (the pmbeg/pmend arrays that
 * gtb_process_block and gtb_block_upload take), valid until gtb_structs_free. */
gtb_status gtb_structs_fields(gtb_structs* b, char** pmbeg, char** pmend);
/* Structure i's description: the path, " Chn:<id>" and " (M:<model>)" as the
 * reference's reader forms it (PMBatchStrData.h:525-545). */
const char* gtb_structs_description(const gtb_structs* b, int i);
void gtb_structs_free(gtb_structs* b);

/* Clustering of n structures from the records of their all-against-all
 * block (queries = references = the n structures, record (q, i) at
 * (q*n + i)*GTB_NOUT), as the reference's clustering writer does it
 * (TdClustWriter.h:225-488, TdClustWriter.cpp:271-414; the --cls options).
 * The distance of structure q to an earlier structure i comes from record
 * (q, i): 1 - TM-score by the --sort measure (or the RMSD), or the largest
 * distance when the aligned residues cover less than `coverage` of either
 * length (of both with `onesided`) or the pair was not aligned.  The
 * pointer representation of single or complete linkage is built over the
 * structures in their order; clusters are cut at the threshold.  Host code:
 * needs no device. */
enum { GTB_LINKAGE_COMPLETE = 0, GTB_LINKAGE_SINGLE = 1 };
/* --sort codes that define the distance (CLOptions.h:64-70) */
enum {
    GTB_SORT_TMGREATER = 0, GTB_SORT_TMREF = 1, GTB_SORT_TMQUERY = 2,
    GTB_SORT_TMHARMONIC = 3, GTB_SORT_RMSD = 4
};
typedef struct {
    int   linkage;     /* --cls-algorithm: 0 complete (default), 1 single */
    int   measure;     /* --sort: GTB_SORT_* (default 0) */
    float threshold;   /* --cls-threshold: TM-score (or RMSD) to join (default 0.5) */
    float coverage;    /* --cls-coverage (0,1] (default 0.7) */
    int   onesided;    /* --cls-one-sided-coverage */
} gtb_cluster_options;

/* Out: pi/lambda (n each, may be NULL): the pointer representation; the
 * clusters: *ncl of them, cluster c's structures at member[offset[c] ..
 * offset[c+1]) (n entries in all; the representative, the member of the
 * smallest lambda, first, then the others in the writer's order), rep[c]
 * its representative (rep and offset sized n and n+1).  The reference's
 * file lists clusters by size, largest first, then by the representative's
 * id. */
gtb_status gtb_cluster(int n, const float* alndata, const int* lens,
                       const gtb_cluster_options* opts, int* pi, float* lambda,
                       int* member, int* offset, int* rep, int* ncl);

/* The same, one structure at a time (O(n) memory, as the reference runs it
 * while query blocks finish): create with the n lengths; add structure q =
 * 0, 1, ..., n-1 in order with rec = its records against structures 0..q-1
 * (rec[i*GTB_NOUT], i < q; a query's row of its all-against-all block);
 * finish once all n are added (outputs as gtb_cluster); destroy. */
typedef struct gtb_clusterer gtb_clusterer;
gtb_status gtb_cluster_create(int n, const int* lens, const gtb_cluster_options* opts,
                              gtb_clusterer** out);
gtb_status gtb_cluster_add(gtb_clusterer* c, int q, const float* rec);
gtb_status gtb_cluster_finish(gtb_clusterer* c, int* pi, float* lambda, int* member,
                              int* offset, int* rep, int* ncl);
void gtb_cluster_destroy(gtb_clusterer* c);

#ifdef __cplusplus
}
#endif
#endif
