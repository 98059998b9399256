// gtb_noalloc.cu -- the search over caller-owned device buffers, with all
// working memory in a fixed static device array.
//
// Why: some callers cannot allocate device memory at the moment they want to
// align structures -- e.g. code running inside another framework's memory
// pool that forbids outside cudaMalloc/cudaFree, a process whose allocator is
// locked while a CUDA graph is being built elsewhere, or a service that must
// keep its device footprint fixed after start-up.  They own their inputs and
// outputs; this entry point needs nothing else from the allocator.
//
// Limits and behaviour:
//  * working memory (pair state, DP traceback words and row buffers, aligned
//    pair lists, per-pair offsets) comes from g_noalloc_scratch below,
//    GTB_NOALLOC_SCRATCH_BYTES = 16 MiB.  Every GPU that loads this library
//    holds that array (and 768 KiB of constant tables) until the process exits.
//    A block whose working memory does not fit, or that has more than
//    GTB_NOALLOC_MAX_PAIRS pairs, is rejected with GTB_ERR_NOMEM and a message
//    before anything runs;
//  * the first call on a device does a one-time set-up on that device (looks
//    up the device addresses of the static arrays and fills the constant
//    tables, with that device current); make that first call before any
//    stream capture;
//  * every call uses the same scratch array and leaves its contents behind.
//    Only the two molecule-type flags must start at zero, and each call
//    clears them first; the pair state is initialised by the first kernel of
//    each call and every other region is written before it is read.  Calls
//    that overlap on the GPU of one device (on different streams, or from
//    different host threads at once) race on that device's scratch array and
//    must not be issued; calls in order on one stream are fine, and so are
//    calls from different host threads on different devices (the host-side
//    plan is per thread);
//  * a block that would pair two nucleic-acid structures is refused with
//    GTB_ERR_UNSUPPORTED, like gtb_process_block refuses it: the molecule
//    types are read back from the device before any search work;
//  * the caller's current device is restored before the call returns;
//  * nothing here calls cudaMalloc, cudaFree or any allocating routine.
#include <cstdio>
#include <cstring>
#include <mutex>
#include <cuda_runtime.h>

#include "gtb200.h"
#include "gtb_kernels.cuh"

using namespace gtb;

namespace {

constexpr size_t SCRATCH_BYTES = (size_t)16 << 20;
constexpr int TBLN = 65536;
constexpr int MAXDEV = 64;

static __device__ __align__(256) unsigned char g_noalloc_scratch[SCRATCH_BYTES];
static __device__ __align__(256) float g_noalloc_d0[TBLN];
static __device__ __align__(256) float g_noalloc_d82[TBLN];
static __device__ __align__(256) float g_noalloc_d0fin[TBLN];

struct DevState {
    bool ready = false;
    unsigned char* scratch = nullptr;
    float *d0 = nullptr, *d82 = nullptr, *d0fin = nullptr;
};
static DevState g_dev[MAXDEV];
static std::mutex g_setup_mutex;
static float h_tbl[3][TBLN];
// Host copies of the per-pair offsets (4 arrays of up to MAX_PAIRS+1 entries)
// and of the back-to-back residue offsets of the (x, y, z, 0) copies.  One set
// per host thread, so that threads calling on different devices at once do
// not overwrite each other's plan before it is copied to the device.
static thread_local long long h_offs[4 * (GTB_NOALLOC_MAX_PAIRS + 1)];
static thread_local int h_coff[2 * (GTB_NOALLOC_MAX_PAIRS + 1)];
// Flag read back after the molecule-type check (per host thread, as above).
static thread_local int h_naflag[2];

// Sets flag[0] when some query is a nucleic acid and flag[1] when some
// reference is; a pair of two nucleic acids is refused by the caller.
__global__ void k_na_check(const int* qmol, int nq, const int* rmol, int nr, int* flag) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < nq) { if (qmol[i] == 1) atomicOr(flag, 1); }
    else if (i < nq + nr) { if (rmol[i - nq] == 1) atomicOr(flag + 1, 1); }
}

// Restores the caller's current device when the call returns.
struct DeviceGuard {
    int prev = -1;
    DeviceGuard() { if (cudaGetDevice(&prev) != cudaSuccess) prev = -1; }
    ~DeviceGuard() { if (prev >= 0) cudaSetDevice(prev); }
};

size_t al256(size_t x) { return (x + 255) & ~(size_t)255; }

// the --pre-similarity screen runs for this block (as in launch setup below)
bool B_presim_on(const gtb_options* o, int qmax, int rmax) {
    return 0.f < o->presimilarity && PRESIM_EDGE < qmax && PRESIM_EDGE < rmax;
}

void setmsg(char* buf, size_t len, const char* fmt, long long a, long long b) {
    if (buf && len) snprintf(buf, len, fmt, a, b);
}

// One-time set-up on the current device: device addresses of the static
// arrays (the host-side names are only stand-ins) and the constant tables.
cudaError_t setup(int dev, cudaStream_t st) {
    std::lock_guard<std::mutex> lk(g_setup_mutex);
    DevState& D = g_dev[dev];
    if (D.ready) return cudaSuccess;
    cudaError_t e;
    if ((e = cudaGetSymbolAddress((void**)&D.scratch, g_noalloc_scratch)) != cudaSuccess) return e;
    if ((e = cudaGetSymbolAddress((void**)&D.d0, g_noalloc_d0)) != cudaSuccess) return e;
    if ((e = cudaGetSymbolAddress((void**)&D.d82, g_noalloc_d82)) != cudaSuccess) return e;
    if ((e = cudaGetSymbolAddress((void**)&D.d0fin, g_noalloc_d0fin)) != cudaSuccess) return e;
    make_tables(h_tbl[0], h_tbl[1], h_tbl[2], TBLN);
    configure_kernels();
    if ((e = cudaMemcpyAsync(D.d0, h_tbl[0], sizeof(h_tbl[0]), cudaMemcpyHostToDevice, st)) != cudaSuccess) return e;
    if ((e = cudaMemcpyAsync(D.d82, h_tbl[1], sizeof(h_tbl[1]), cudaMemcpyHostToDevice, st)) != cudaSuccess) return e;
    if ((e = cudaMemcpyAsync(D.d0fin, h_tbl[2], sizeof(h_tbl[2]), cudaMemcpyHostToDevice, st)) != cudaSuccess) return e;
    if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return e;
    D.ready = true;
    return cudaSuccess;
}

}  // namespace

extern "C" gtb_status gtb_process_block_noalloc(int device, const gtb_options* opts, float scorethld,
                                                const gtb_dev_soa* q, const gtb_dev_soa* r,
                                                float* d_alndata, float* d_tfm, float* d_numerr,
                                                void* stream, char* errbuf, size_t errlen) {
    if (errbuf && errlen) errbuf[0] = 0;
    if (!opts || !q || !r || !d_alndata || !d_tfm || device < 0 || device >= MAXDEV) {
        setmsg(errbuf, errlen, "null argument or device out of range (%lld, %lld)", device, MAXDEV);
        return GTB_ERR_ARG;
    }
    if (!opts->nodetailedsearch || opts->clsfilter) {
        setmsg(errbuf, errlen, "the detailed search (%lld) and the clustering prefilter (%lld) are not implemented here",
               !opts->nodetailedsearch, (long long)opts->clsfilter);
        return GTB_ERR_UNSUPPORTED;
    }
    if (!(scorethld >= 0.f && scorethld < 1.f) || opts->depth < 0 || opts->depth > 3 ||
        opts->refinement < GTB_REFINEMENT_LOG || opts->refinement > GTB_REFINEMENT_FULLA ||
        opts->convergence < 1 || opts->convergence > 30 || !(opts->prescore >= 0.f && opts->prescore < 1.f) ||
        opts->polish_steps < 0 || opts->polish_steps > 50 ||
        !(opts->presimilarity >= 0.f && opts->presimilarity < 1e6f)) {
        setmsg(errbuf, errlen, "option out of range (%lld %lld)", 0, 0);
        return GTB_ERR_ARG;
    }
    if (q->n < 1 || r->n < 1 || !q->lens || !r->lens || !q->d_lens || !r->d_lens || !q->d_offs ||
        !r->d_offs || !q->d_mol || !r->d_mol || !q->d_x || !q->d_y || !q->d_z || !r->d_x ||
        !r->d_y || !r->d_z || !q->d_rsd || !r->d_rsd || !q->d_ss || !r->d_ss) {
        setmsg(errbuf, errlen, "empty block or null field (%lld x %lld)", q->n, r->n);
        return GTB_ERR_ARG;
    }
    long long npairs = (long long)q->n * r->n;
    if (npairs > GTB_NOALLOC_MAX_PAIRS) {
        setmsg(errbuf, errlen, "block has %lld pairs; the allocation-free entry point takes at most %lld",
               npairs, GTB_NOALLOC_MAX_PAIRS);
        return GTB_ERR_NOMEM;
    }
    int qmax = 0, qmin = 1 << 30, rmax = 0, rmin = 1 << 30;
    for (int i = 0; i < q->n; i++) {
        int L = q->lens[i];
        if (L < 1 || L > 65535) { setmsg(errbuf, errlen, "query %lld has length %lld", i, L); return L > 65535 ? GTB_ERR_TOO_LONG : GTB_ERR_ARG; }
        qmax = L > qmax ? L : qmax; qmin = L < qmin ? L : qmin;
    }
    for (int i = 0; i < r->n; i++) {
        int L = r->lens[i];
        if (L < 1 || L > 65535) { setmsg(errbuf, errlen, "reference %lld has length %lld", i, L); return L > 65535 ? GTB_ERR_TOO_LONG : GTB_ERR_ARG; }
        rmax = L > rmax ? L : rmax; rmin = L < rmin ? L : rmin;
    }
    // plan the scratch: pair state, offsets, traceback, DP rows, aligned pairs
    int np = (int)npairs;
    long long* obt = h_offs;
    long long* orow = h_offs + (np + 1);
    long long* oaln = h_offs + 2 * (np + 1);
    long long* ostr = h_offs + 3 * (np + 1);
    obt[0] = orow[0] = oaln[0] = ostr[0] = 0;
    for (int i = 0; i < np; i++) {
        int lq = q->lens[i / r->n], lr = r->lens[i % r->n];
        obt[i + 1] = obt[i] + gtb::bt_words(lq, lr);
        orow[i + 1] = orow[i] + lr;
        oaln[i + 1] = oaln[i] + (lq < lr ? lq : lr);
        ostr[i + 1] = 0;
    }
    size_t sz = 0;
    auto carve = [&](size_t bytes) { size_t o = sz; sz += al256(bytes); return o; };
    size_t o_ints = carve((size_t)np * 8 * sizeof(int));
    size_t o_flts = carve((size_t)np * 4 * sizeof(float));
    size_t o_tib = carve((size_t)np * 12 * sizeof(float));
    size_t o_tgr = carve((size_t)np * 12 * sizeof(float));
    size_t o_out = carve((size_t)np * 16 * sizeof(float));
    size_t o_err = carve((size_t)np * 4 * sizeof(float));
    size_t o_offs = carve((size_t)(np + 1) * 4 * sizeof(long long));
    size_t o_bt = carve((size_t)obt[np] * sizeof(unsigned));
    size_t o_row = carve((size_t)orow[np] * sizeof(float));
    size_t o_aln = carve((size_t)oaln[np] * sizeof(unsigned));
    size_t o_alc = carve((size_t)oaln[np] * 6 * sizeof(float));
    long long qres = 0, rres = 0;
    for (int i = 0; i < q->n; i++) { h_coff[i] = (int)qres; qres += q->lens[i]; }
    for (int i = 0; i < r->n; i++) { h_coff[q->n + i] = (int)rres; rres += r->lens[i]; }
    size_t o_q4 = carve((size_t)qres * sizeof(float4));
    size_t o_r4 = carve((size_t)rres * sizeof(float4));
    size_t o_co = carve((size_t)(q->n + r->n) * sizeof(int));
    size_t o_rl = carve((size_t)np * sizeof(int));
    size_t o_rh = carve((size_t)4097 * sizeof(int));
    size_t o_na = carve(2 * sizeof(int));
    if (sz > SCRATCH_BYTES) {
        setmsg(errbuf, errlen, "block needs %lld bytes of working memory; the static scratch holds %lld",
               (long long)sz, (long long)SCRATCH_BYTES);
        return GTB_ERR_NOMEM;
    }

    cudaStream_t st = (cudaStream_t)stream;
    DeviceGuard keep_device;
    cudaError_t e = cudaSetDevice(device);
    if (e == cudaSuccess) e = setup(device, st);
    if (e != cudaSuccess) {
        if (errbuf && errlen) snprintf(errbuf, errlen, "set-up: %s", cudaGetErrorString(e));
        return GTB_ERR_CUDA;
    }
    const DevState& D = g_dev[device];
    unsigned char* base = D.scratch;

    // The molecule types are device data: look at them before any work, and
    // refuse a block that would pair two nucleic-acid structures (the search
    // here scores with protein rules only), as gtb_process_block does.
    {
        int* naf = (int*)(base + o_na);
        e = cudaMemsetAsync(naf, 0, 2 * sizeof(int), st);
        if (e == cudaSuccess) {
            int nt = q->n + r->n;
            k_na_check<<<(nt + 255) / 256, 256, 0, st>>>(q->d_mol, q->n, r->d_mol, r->n, naf);
            e = cudaGetLastError();
        }
        if (e == cudaSuccess) e = cudaMemcpyAsync(h_naflag, naf, sizeof(h_naflag), cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) {
            if (errbuf && errlen) snprintf(errbuf, errlen, "molecule-type check: %s", cudaGetErrorString(e));
            return GTB_ERR_CUDA;
        }
        if ((h_naflag[0] && h_naflag[1]) || (B_presim_on(opts, qmax, rmax) && (h_naflag[0] || h_naflag[1]))) {
            setmsg(errbuf, errlen, "nucleic-acid structure pairs are not supported (%lld, %lld)",
                   h_naflag[0], h_naflag[1]);
            return GTB_ERR_UNSUPPORTED;
        }
    }

    Blk B{};
    B.nq = q->n; B.nr = r->n;
    B.qlen = q->d_lens; B.rlen = r->d_lens; B.qoff = q->d_offs; B.roff = r->d_offs;
    B.qx = q->d_x; B.qy = q->d_y; B.qz = q->d_z; B.rx = r->d_x; B.ry = r->d_y; B.rz = r->d_z;
    int* coff = (int*)(base + o_co);
    B.q4 = (const float4*)(base + o_q4); B.r4 = (const float4*)(base + o_r4);
    B.q4off = coff; B.r4off = coff + q->n;
    B.qa = q->d_rsd; B.ra = r->d_rsd; B.qs = q->d_ss; B.rs = r->d_ss;
    B.qmol = q->d_mol; B.rmol = r->d_mol;
    B.qmax = qmax; B.qmin = qmin; B.rmax = rmax; B.rmin = rmin;
    B.t_d0 = D.d0; B.t_d82 = D.d82; B.t_d0fin = D.d0fin;
    B.stepinit = (opts->depth == 3) ? 5 : 1;
    B.refinement = opts->refinement; B.depth = opts->depth; B.twotm = opts->twotmscore ? 1 : 0;
    B.addss = opts->addsearchbyss ? 1 : 0;
    B.presim = B_presim_on(opts, qmax, rmax) ? opts->presimilarity : 0.f;
    B.symmetric = opts->symmetric; B.nodeletions = opts->nodeletions;

    Bat T{};
    T.p0 = 0; T.np = np;
    int* ints = (int*)(base + o_ints);
    T.flags = ints; T.seedq = ints + np; T.seedr = ints + 2 * np; T.naln = ints + 3 * np;
    T.sfndx = ints + 4 * np; T.sfpos = ints + 5 * np; T.sfndx_cur = ints + 6 * np; T.sfpos_cur = ints + 7 * np;
    float* fl = (float*)(base + o_flts);
    T.grand = fl; T.best = fl + np; T.best0 = fl + 2 * np; T.rmsd32 = fl + 3 * np;
    T.tfm_ib = (float*)(base + o_tib); T.tfm_gr = (float*)(base + o_tgr);
    T.out = (float*)(base + o_out); T.err = (float*)(base + o_err);
    long long* offs = (long long*)(base + o_offs);
    T.off_bt = offs; T.off_row = offs + (np + 1); T.off_aln = offs + 2 * (np + 1); T.off_str = offs + 3 * (np + 1);
    T.bt = (unsigned*)(base + o_bt); T.row = (float*)(base + o_row);
    T.aln = (unsigned*)(base + o_aln); T.str = nullptr;
    T.alc = (float*)(base + o_alc);
    T.rlist = (int*)(base + o_rl); T.rhist = (int*)(base + o_rh);
    T.nff = np; T.ff_pair = nullptr; T.ff_chunk = nullptr; T.ff_nch = nullptr; T.ff_key = nullptr;
    T.launches = nullptr;
    T.alt_rci = -1;

    // the host offsets are copied from the static host array (no allocation)
    e = cudaMemcpyAsync(offs, h_offs, (size_t)(np + 1) * 4 * sizeof(long long), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(coff, h_coff, (size_t)(q->n + r->n) * sizeof(int), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) {
        long long nl = 0;
        launch_pack4_structs((float4*)(base + o_q4), q->d_x, q->d_y, q->d_z, q->d_offs, q->d_lens, coff, q->n, st);
        launch_pack4_structs((float4*)(base + o_r4), r->d_x, r->d_y, r->d_z, r->d_offs, r->d_lens, coff + q->n, r->n, st);
        launch_secstr(q->d_ss, q->d_x, q->d_y, q->d_z, q->d_lens, q->d_offs, q->d_mol, q->n, st, &nl);
        launch_secstr(r->d_ss, r->d_x, r->d_y, r->d_z, r->d_lens, r->d_offs, r->d_mol, r->n, st, &nl);
        launch_stages(B, T, opts->refinement, opts->depth, opts->convergence, opts->prescore,
                      opts->referenced, scorethld, st, nullptr, opts->polish_steps);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(d_alndata, T.out, (size_t)np * 16 * sizeof(float), cudaMemcpyDeviceToDevice, st);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(d_tfm, T.tfm_gr, (size_t)np * 12 * sizeof(float), cudaMemcpyDeviceToDevice, st);
    if (e == cudaSuccess && d_numerr)
        e = cudaMemcpyAsync(d_numerr, T.err, (size_t)np * 4 * sizeof(float), cudaMemcpyDeviceToDevice, st);
    // the host offsets array is reused by the next call: wait for its copy
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) {
        if (errbuf && errlen) snprintf(errbuf, errlen, "%s", cudaGetErrorString(e));
        return GTB_ERR_CUDA;
    }
    return GTB_OK;
}
