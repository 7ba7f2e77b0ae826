// sim.cu - the single-shot C ABI (bp_sim) and the reference-format writers.
#include <sys/stat.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "runner.h"

namespace bpk {
const char* last_error_cstr();
}
using namespace bpk;

struct bp_sim {
    Shot shot;
    Runner run;
    cudaStream_t st = nullptr;
    int device = 0;
    double cfl_dtmax = 0;          // the stability limit found at create (check_cfl), 0 = not checked
    float* d_zf = nullptr;         // variable z grid: the factor tables (arena cache)
    size_t d_zf_bytes = 0;
};

#define SIM_CK(call)                                                                       \
    do {                                                                                   \
        cudaError_t e_ = (call);                                                           \
        if (e_ != cudaSuccess) {                                                           \
            set_error(std::string(#call) + ": " + cudaGetErrorString(e_));                 \
            return e_ == cudaErrorMemoryAllocation ? BP_ERR_OOM : BP_ERR_CUDA;             \
        }                                                                                  \
    } while (0)

// Checkpoint image: this header, then the shot's state regions in the order
// Shot::state_regions lists them.
struct CkptHeader {
    char magic[8];
    int32_t version, precision, dim, order, nx, ny, nz, nt, nurec, it, nregions, pad;
    uint64_t payload;
};
static const char kCkptMagic[8] = {'B', 'P', 'C', 'K', 'P', 'T', '0', '1'};

// Binary output file: this header, then the float32 array, little-endian,
// last dimension fastest.
struct BinHeader {
    char magic[8];
    int32_t version, dtype, ndims, dims[3];
};
static const char kBinMagic[8] = {'B', 'P', 'B', 'I', 'N', '0', '0', '1'};

static const char* kFieldNames[BP_NFIELDS] = {"vux", "vuy", "vuz", "vwx", "vwy", "vwz", "p",
                                              "txx", "tyy", "tzz", "txy", "txz", "tyz"};

static int check_device(int device) {
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess || n <= 0) {
        cudaGetLastError();
        set_error(std::string("no CUDA device: ") + cudaGetErrorString(e));
        return BP_ERR_NO_DEVICE;
    }
    if (device < 0 || device >= n) { set_error("device ordinal out of range"); return BP_ERR_ARG; }
    // two attribute queries: cudaGetDeviceProperties fills every field and took
    // 5-60 ms per call, inside every bp_create
    int major = 0, minor = 0;
    if (cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, device) != cudaSuccess ||
        cudaDeviceGetAttribute(&minor, cudaDevAttrComputeCapabilityMinor, device) != cudaSuccess) {
        cudaGetLastError();
        set_error("cannot query the device's compute capability");
        return BP_ERR_NO_DEVICE;
    }
    if (major != 10) {
        set_error("this library is built for sm_100a (B200); device is sm_" + std::to_string(major) + std::to_string(minor));
        return BP_ERR_NO_DEVICE;
    }
    return BP_OK;
}

extern "C" {

const char* bp_error_string(int code) {
    switch (code) {
        case BP_OK: return "ok";
        case BP_ERR_ARG: return "invalid argument";
        case BP_ERR_OOM: return "out of memory";
        case BP_ERR_CUDA: return "CUDA error";
        case BP_ERR_CFL: return "time step violates the stability limit";
        case BP_ERR_UNSTABLE: return "non-finite wavefield";
        case BP_ERR_TIMEOUT: return "timed out";
        case BP_ERR_STATE: return "invalid state";
        case BP_ERR_NOT_FOUND: return "not found";
        case BP_ERR_NO_DEVICE: return "no usable CUDA device";
        case BP_ERR_BUDGET: return "request exceeds the HBM budget";
        default: return "unknown error";
    }
}
const char* bp_last_error(void) { return last_error_cstr(); }

int bp_debug_fail_allocation(int nth) {
    if (nth < 0) { set_error("nth must be >= 0"); return BP_ERR_ARG; }
    arm_allocation_failure(nth);
    return BP_OK;
}

int bp_create(const bp_config* cfg, const bp_medium* medium, bp_sim** out) {
    if (!out) { set_error("null output pointer"); return BP_ERR_ARG; }
    *out = nullptr;
    int rc = validate_config(cfg);
    if (rc) return rc;
    rc = check_device(cfg->device);
    if (rc) return rc;
    // The stability check scans the host medium on host threads while this
    // thread sets up the device (medium upload, precompute kernels); both only
    // read the medium.  A failing check undoes the set-up.
    double dtmax = 0, vmax = 0;
    int cfl_rc = BP_OK;
    std::thread cfl;
    if (cfg->check_cfl && medium)
        cfl = std::thread([&] { cfl_rc = bp_cfl_limit(cfg, medium, &dtmax, &vmax); });
    // joins the scan; reports its failure unless an earlier one is being returned
    auto cfl_verdict = [&](bool report) -> int {
        if (!cfl.joinable()) return BP_OK;
        cfl.join();
        if (!report) return BP_OK;
        if (cfl_rc) { set_error("stability check: bad medium arrays"); return cfl_rc; }
        if ((double)cfg->dt > dtmax) {
            char buf[160];
            snprintf(buf, sizeof buf, "dt=%g exceeds the stability limit %g (vmax=%g m/s)", (double)cfg->dt, dtmax, vmax);
            set_error(buf);
            return BP_ERR_CFL;
        }
        return BP_OK;
    };
    cudaError_t e = cudaSetDevice(cfg->device);
    if (e != cudaSuccess) { cfl_verdict(false); set_error(cudaGetErrorString(e)); return BP_ERR_CUDA; }
    bp_sim* s = new bp_sim();
    s->device = cfg->device;
    e = cudaStreamCreateWithFlags(&s->st, cudaStreamNonBlocking);
    if (e != cudaSuccess) { cfl_verdict(false); set_error(cudaGetErrorString(e)); delete s; return BP_ERR_CUDA; }
    rc = s->shot.create(cfg, medium, s->st);
    const int crc = cfl_verdict(rc == BP_OK);
    if (!rc && crc) { cudaStreamSynchronize(s->st); rc = crc; }
    s->cfl_dtmax = cfg->check_cfl && medium ? dtmax : 0.0;
    if (rc) { s->shot.destroy(); cudaStreamDestroy(s->st); delete s; return rc; }
    s->run.post_in_t = s->shot.post_in_t;
    s->run.rounding = cfg->rounding;
    s->run.ntiles_f = s->shot.ntiles_f;
    s->run.nitems_i = s->shot.nitems_i;
    s->run.indexed = s->shot.med_tuples > 0;
    s->run.nbands_i = s->shot.desc.nbands_i;
    s->run.configure(cfg->precision, cfg->dim, cfg->order, s->shot.d_desc, 1, s->shot.ntiles, s->shot.ntiles_s,
                     s->shot.ntiles_m, s->shot.nurec, s->st, 0, 32);
    *out = s;
    return BP_OK;
}

int bp_run(bp_sim* s, int nsteps) {
    if (!s || nsteps < 0) { set_error("bad arguments"); return BP_ERR_ARG; }
    SIM_CK(cudaSetDevice(s->device));
    Shot& sh = s->shot;
    while (nsteps > 0 && sh.it_host < sh.cfg.nt) {
        int m = std::min(nsteps, sh.cfg.nt - sh.it_host);
        int next_snap = -1;
        for (int st : sh.snap_steps)
            if (st >= sh.it_host && (next_snap < 0 || st < next_snap)) next_snap = st;
        if (next_snap >= 0) m = std::min(m, next_snap - sh.it_host + 1);
        SIM_CK(s->run.run(m));
        sh.it_host += m;
        const int done_it = sh.it_host - 1;
        for (int k = 0; k < (int)sh.snap_steps.size(); k++) {
            if (sh.snap_steps[k] != done_it) continue;
            for (int f = 0; f < BP_NFIELDS; f++) {
                long long off = sh.snap_off[(size_t)k * BP_NFIELDS + f];
                if (off < 0) continue;
                int sy = (sh.cfg.dim == 3 && sh.cfg.snap_y >= 0) ? sh.cfg.snap_y : -1;
                SIM_CK(launch_snapshot(sh.cfg.precision, sh.d_desc, 0, f, sy, sh.d_snap + off, done_it, s->st));
            }
        }
        nsteps -= m;
    }
    return BP_OK;
}

int bp_run_timed(bp_sim* s, int nsteps, float* ms) {
    if (!s || !ms) { set_error("bad arguments"); return BP_ERR_ARG; }
    SIM_CK(cudaSetDevice(s->device));
    cudaEvent_t a, b;
    SIM_CK(cudaEventCreate(&a));
    SIM_CK(cudaEventCreate(&b));
    cudaEventRecord(a, s->st);
    int rc = bp_run(s, nsteps);
    cudaEventRecord(b, s->st);
    cudaError_t e = cudaEventSynchronize(b);
    float t = 0;
    if (e == cudaSuccess) e = cudaEventElapsedTime(&t, a, b);
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    if (rc) return rc;
    if (e != cudaSuccess) { set_error(cudaGetErrorString(e)); return BP_ERR_CUDA; }
    *ms = t;
    return BP_OK;
}

int bp_sync(bp_sim* s) {
    if (!s) { set_error("null sim"); return BP_ERR_ARG; }
    SIM_CK(cudaStreamSynchronize(s->st));
    int rc = s->run.device_error();
    if (rc) { set_error("a step kernel gave up waiting (staged tile copies or interleaved band counters)"); return rc; }
    const int bad = s->shot.blowup_step(s->st);
    if (bad) {
        set_error("non-finite value recorded at a receiver at step " + std::to_string(bad - 1) +
                  " (dt above the stability limit?)");
        return BP_ERR_UNSTABLE;
    }
    return BP_OK;
}

int bp_set_graph_steps(bp_sim* s, int steps) {
    if (!s || steps < 0) { set_error("bad arguments"); return BP_ERR_ARG; }
    SIM_CK(cudaStreamSynchronize(s->st));
    s->run.graph_steps = steps;
    s->run.reset_graph();
    return BP_OK;
}

int bp_set_kernel(bp_sim* s, int variant) {
    if (!s || variant < BP_KERNEL_AUTO || variant > BP_KERNEL_INTERLEAVED) { set_error("bad arguments"); return BP_ERR_ARG; }
    if (variant == BP_KERNEL_FUSED && (s->shot.ntiles_f <= 0 || s->shot.cfg.rounding != BP_ROUND_FAST)) {
        set_error("the fused step kernel covers 2D FP32 and COMP16 with fast rounding, receivers and source "
                  "inside the stencil border");
        return BP_ERR_ARG;
    }
    if (variant == BP_KERNEL_STAGED && !staged_supported(s->shot.cfg.precision, s->shot.cfg.dim)) {
        set_error("the staged kernels cover 2D FP32 and COMP16 only");
        return BP_ERR_ARG;
    }
    if (variant == BP_KERNEL_MARCH && !march_supported(s->shot.cfg.precision, s->shot.cfg.dim)) {
        set_error("the marching kernels cover 2D FP32 and COMP16 only");
        return BP_ERR_ARG;
    }
    if (variant == BP_KERNEL_INTERLEAVED && (s->shot.nitems_i <= 0 || !s->run.d_ctl || !s->run.d_err)) {
        set_error("the interleaved step kernel has no control block for this simulation");
        return BP_ERR_ARG;
    }
    if (s->run.graded && variant != BP_KERNEL_AUTO && variant != BP_KERNEL_REGISTER) {
        set_error("a variable z grid runs the register tile kernels only");
        return BP_ERR_ARG;
    }
    if ((variant == BP_KERNEL_STAGED || variant == BP_KERNEL_MARCH) && s->shot.med_tuples > 0) {
        set_error("the staged and marching kernels read the per-cell coefficient arrays: create the shot with "
                  "medium = BP_MEDIUM_DENSE");
        return BP_ERR_ARG;
    }
    if ((variant == BP_KERNEL_STAGED || variant == BP_KERNEL_MARCH) && s->shot.cfg.rounding != BP_ROUND_FAST) {
        set_error("reference rounding runs the register tile kernels only");
        return BP_ERR_ARG;
    }
    SIM_CK(cudaStreamSynchronize(s->st));
    s->run.variant = variant;
    s->run.select_kernels();
    s->run.reset_graph();
    return BP_OK;
}

int bp_get_step(bp_sim* s, int* it) {
    if (!s || !it) { set_error("bad arguments"); return BP_ERR_ARG; }
    *it = s->shot.it_host;
    return BP_OK;
}

int bp_get_traces(bp_sim* s, int comp, float* host, size_t n) {
    if (!s || !host || comp < 0 || comp >= BP_NTRACE) { set_error("bad arguments"); return BP_ERR_ARG; }
    Shot& sh = s->shot;
    const size_t nt = sh.cfg.nt, nr = sh.cfg.nrec;
    if (n < nr * nt) { set_error("host buffer too small"); return BP_ERR_ARG; }
    SIM_CK(cudaStreamSynchronize(s->st));
    SIM_CK(sh.copy_traces(comp, host));
    return BP_OK;
}

int bp_release_cached_memory(int device) {
    if (device < -1) { set_error("bad device"); return BP_ERR_ARG; }
    release_cached_arenas(device);
    return BP_OK;
}

int bp_receiver_map(bp_sim* s, int* nurec, int* map) {
    if (!s || !nurec) { set_error("bad arguments"); return BP_ERR_ARG; }
    *nurec = s->shot.nurec;
    if (map) for (int r = 0; r < s->shot.cfg.nrec; r++) map[r] = s->shot.urec_of[r];
    return BP_OK;
}

int bp_copy_traces_async(bp_sim* s, int comp, int it0, int n, float* host) {
    if (!s || !host || comp < 0 || comp >= BP_NTRACE || it0 < 0 || n < 0 || it0 + n > s->shot.cfg.nt) {
        set_error("bad arguments");
        return BP_ERR_ARG;
    }
    Shot& sh = s->shot;
    if (n == 0 || sh.nurec == 0) return BP_OK;
    const size_t nt = sh.cfg.nt;
    SIM_CK(cudaSetDevice(s->device));
    SIM_CK(cudaMemcpy2DAsync(host, (size_t)n * 4, sh.desc.traces + (size_t)comp * sh.nurec * nt + it0, nt * 4,
                             (size_t)n * 4, sh.nurec, cudaMemcpyDeviceToHost, s->st));
    return BP_OK;
}

int bp_checkpoint_size(bp_sim* s, size_t* bytes) {
    if (!s || !bytes) { set_error("bad arguments"); return BP_ERR_ARG; }
    size_t n = sizeof(CkptHeader);
    for (auto& r : s->shot.state_regions()) n += r.second;
    *bytes = n;
    return BP_OK;
}

static void ckpt_header(bp_sim* s, CkptHeader& h) {
    const Shot& sh = s->shot;
    std::memset(&h, 0, sizeof h);
    std::memcpy(h.magic, kCkptMagic, 8);
    h.version = 1;
    h.precision = sh.cfg.precision; h.dim = sh.cfg.dim; h.order = sh.cfg.order;
    h.nx = sh.desc.nx; h.ny = sh.desc.ny; h.nz = sh.desc.nz; h.nt = sh.cfg.nt; h.nurec = sh.nurec;
    h.it = sh.it_host;
    const auto regs = sh.state_regions();
    h.nregions = (int)regs.size();
    for (auto& r : regs) h.payload += r.second;
}

int bp_checkpoint(bp_sim* s, void* host, size_t bytes) {
    if (!s || !host) { set_error("bad arguments"); return BP_ERR_ARG; }
    size_t need = 0;
    bp_checkpoint_size(s, &need);
    if (bytes < need) { set_error("checkpoint buffer too small"); return BP_ERR_ARG; }
    SIM_CK(cudaSetDevice(s->device));
    SIM_CK(cudaStreamSynchronize(s->st));
    int rc = s->run.device_error();
    if (rc) { set_error("a phase kernel recorded an error"); return rc; }
    CkptHeader h;
    ckpt_header(s, h);
    std::memcpy(host, &h, sizeof h);
    char* p = static_cast<char*>(host) + sizeof h;
    for (auto& r : s->shot.state_regions()) {
        SIM_CK(cudaMemcpyAsync(p, r.first, r.second, cudaMemcpyDeviceToHost, s->st));
        p += r.second;
    }
    SIM_CK(cudaStreamSynchronize(s->st));
    return BP_OK;
}

int bp_restore(bp_sim* s, const void* host, size_t bytes) {
    if (!s || !host || bytes < sizeof(CkptHeader)) { set_error("bad arguments"); return BP_ERR_ARG; }
    CkptHeader h, mine;
    std::memcpy(&h, host, sizeof h);
    ckpt_header(s, mine);
    if (std::memcmp(h.magic, kCkptMagic, 8) != 0 || h.version != 1) { set_error("not a checkpoint image"); return BP_ERR_ARG; }
    if (h.precision != mine.precision || h.dim != mine.dim || h.order != mine.order || h.nx != mine.nx ||
        h.ny != mine.ny || h.nz != mine.nz || h.nt != mine.nt || h.nurec != mine.nurec ||
        h.nregions != mine.nregions || h.payload != mine.payload) {
        set_error("checkpoint was taken from a simulation of another configuration");
        return BP_ERR_ARG;
    }
    if (bytes < sizeof h + h.payload) { set_error("checkpoint image truncated"); return BP_ERR_ARG; }
    if (h.it < 0 || h.it > h.nt) { set_error("checkpoint step out of range"); return BP_ERR_ARG; }
    SIM_CK(cudaSetDevice(s->device));
    SIM_CK(cudaStreamSynchronize(s->st));
    const char* p = static_cast<const char*>(host) + sizeof h;
    for (auto& r : s->shot.state_regions()) {
        SIM_CK(cudaMemcpyAsync(r.first, p, r.second, cudaMemcpyHostToDevice, s->st));
        p += r.second;
    }
    const int it = h.it;
    SIM_CK(cudaMemcpyAsync(s->shot.desc.step_base, &it, sizeof(int), cudaMemcpyHostToDevice, s->st));
    SIM_CK(cudaStreamSynchronize(s->st));
    s->shot.it_host = it;
    return BP_OK;
}

int bp_snapshot_size(bp_sim* s, size_t* n) {
    if (!s || !n) { set_error("bad arguments"); return BP_ERR_ARG; }
    *n = s->shot.snap_n;
    return BP_OK;
}

int bp_get_snapshot(bp_sim* s, int k, int field, float* host, size_t n) {
    if (!s || !host || field < 0 || field >= BP_NFIELDS) { set_error("bad arguments"); return BP_ERR_ARG; }
    Shot& sh = s->shot;
    if (k < 0 || k >= (int)sh.snap_steps.size()) { set_error("no such snapshot"); return BP_ERR_NOT_FOUND; }
    long long off = sh.snap_off[(size_t)k * BP_NFIELDS + field];
    if (off < 0) { set_error("field not captured at this snapshot"); return BP_ERR_NOT_FOUND; }
    if (sh.it_host <= sh.snap_steps[k]) { set_error("snapshot step not reached yet"); return BP_ERR_STATE; }
    if (n < sh.snap_n) { set_error("host buffer too small"); return BP_ERR_ARG; }
    SIM_CK(cudaStreamSynchronize(s->st));
    SIM_CK(cudaMemcpy(host, sh.d_snap + off, sh.snap_n * 4, cudaMemcpyDeviceToHost));
    return BP_OK;
}

int bp_get_dims(bp_sim* s, int* nxe, int* nye, int* nze) {
    if (!s) { set_error("null sim"); return BP_ERR_ARG; }
    if (nxe) *nxe = s->shot.desc.nx;
    if (nye) *nye = s->shot.desc.ny;
    if (nze) *nze = s->shot.desc.nz;
    return BP_OK;
}

int bp_get_field_f64(bp_sim* s, int field, double* host, size_t n) {
    if (!s || !host || field < 0 || field >= BP_NFIELDS) { set_error("bad arguments"); return BP_ERR_ARG; }
    Shot& sh = s->shot;
    if (!sh.desc.f[field]) { set_error("field not evolved in this dimension"); return BP_ERR_NOT_FOUND; }
    const size_t cnt = (size_t)sh.desc.nx * sh.desc.ny * sh.desc.nz;
    if (n < cnt) { set_error("host buffer too small"); return BP_ERR_ARG; }
    SIM_CK(cudaSetDevice(s->device));
    double* d = nullptr;
    SIM_CK(cudaMalloc(&d, cnt * 8));
    cudaError_t e = launch_field_f64(sh.cfg.precision, sh.d_desc, field, d, s->st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(host, d, cnt * 8, cudaMemcpyDeviceToHost, s->st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s->st);
    cudaFree(d);
    if (e != cudaSuccess) { set_error(cudaGetErrorString(e)); return BP_ERR_CUDA; }
    return BP_OK;
}

int bp_get_field(bp_sim* s, int field, float* host, size_t n) {
    if (!s || !host) { set_error("bad arguments"); return BP_ERR_ARG; }
    const size_t cnt = (size_t)s->shot.desc.nx * s->shot.desc.ny * s->shot.desc.nz;
    if (n < cnt) { set_error("host buffer too small"); return BP_ERR_ARG; }
    std::vector<double> tmp(cnt);
    int rc = bp_get_field_f64(s, field, tmp.data(), cnt);
    if (rc) return rc;
    for (size_t i = 0; i < cnt; i++) host[i] = (float)tmp[i];
    return BP_OK;
}

int bp_get_coef(bp_sim* s, int which, float* host, size_t n) {
    if (!s || !host || which < 0 || which >= VC_COUNT + TC_COUNT) { set_error("bad arguments"); return BP_ERR_ARG; }
    Shot& sh = s->shot;
    const size_t cnt = (size_t)sh.desc.nx * sh.desc.ny * sh.desc.nz;
    if (n < cnt) { set_error("host buffer too small"); return BP_ERR_ARG; }
    SIM_CK(cudaSetDevice(s->device));
    float* d = nullptr;
    SIM_CK(cudaMalloc(&d, cnt * 4));
    cudaError_t e = launch_coef(sh.cfg.precision, sh.d_desc, which, d, s->st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(host, d, cnt * 4, cudaMemcpyDeviceToHost, s->st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s->st);
    cudaFree(d);
    if (e != cudaSuccess) { set_error(cudaGetErrorString(e)); return BP_ERR_CUDA; }
    return BP_OK;
}

int bp_field_energy(bp_sim* s, double* energy) {
    if (!s || !energy) { set_error("bad arguments"); return BP_ERR_ARG; }
    SIM_CK(cudaSetDevice(s->device));
    Shot& sh = s->shot;
    SIM_CK(launch_energy(sh.cfg.precision, sh.d_desc, sh.d_scratch, sh.d_out, s->st));
    SIM_CK(cudaMemcpyAsync(energy, sh.d_out, sizeof(double), cudaMemcpyDeviceToHost, s->st));
    SIM_CK(cudaStreamSynchronize(s->st));
    return BP_OK;
}

int bp_get_scaling(bp_sim* s, int* em, int* es, float* dyn_scale, double* kmax, double* rmax) {
    if (!s) { set_error("null sim"); return BP_ERR_ARG; }
    Shot& sh = s->shot;
    if (em) *em = sh.em;
    if (es) *es = sh.es;
    if (dyn_scale) {
        int it = sh.it_host;
        *dyn_scale = sh.dyn.empty() ? 1.0f : sh.dyn[it > 0 ? std::min(it - 1, (int)sh.dyn.size() - 1) : 0];
    }
    if (kmax) *kmax = sh.kmax;
    if (rmax) *rmax = sh.rmax;
    return BP_OK;
}

// Per-launch device times from events recorded around every launch of the
// profiled steps, read after one synchronisation at the end: a wait per step
// would leave the GPU idle between steps and time each launch from idle.
struct EventRing {
    std::vector<cudaEvent_t> ev;
    ~EventRing() { for (auto e : ev) cudaEventDestroy(e); }
    cudaError_t make(size_t n) {
        ev.resize(n, nullptr);
        for (auto& e : ev) { cudaError_t r = cudaEventCreate(&e); if (r != cudaSuccess) return r; }
        return cudaSuccess;
    }
};

int bp_profile_phases(bp_sim* s, int nsteps, float ms[3]) {
    if (!s || !ms || nsteps < 1) { set_error("bad arguments"); return BP_ERR_ARG; }
    SIM_CK(cudaSetDevice(s->device));
    Shot& sh = s->shot;
    Runner& R = s->run;
    nsteps = std::min(nsteps, sh.cfg.nt - sh.it_host);
    if (nsteps < 1) { set_error("no steps left to profile"); return BP_ERR_STATE; }
    EventRing E;
    SIM_CK(E.make((size_t)4 * nsteps));
    cudaError_t e = cudaSuccess;
    for (int i = 0; i < nsteps && e == cudaSuccess; i++) {
        cudaEvent_t* ev = &E.ev[4 * i];
        cudaEventRecord(ev[0], s->st);
        e = R.phase(true, 0);
        cudaEventRecord(ev[1], s->st);
        if (e == cudaSuccess) e = R.phase(false, 0);
        cudaEventRecord(ev[2], s->st);
        if (e == cudaSuccess && !R.fused_post()) e = launch_post(R.prec, R.d_shots, R.nshots, R.max_rec, 0, 1, s->st);
        if (e == cudaSuccess) e = launch_advance(R.d_shots, R.nshots, 1, s->st);
        cudaEventRecord(ev[3], s->st);
        R.launches += R.launches_per_step() + 1;
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(s->st);
    if (e != cudaSuccess) { set_error(cudaGetErrorString(e)); return BP_ERR_CUDA; }
    double acc[3] = {0, 0, 0};
    for (int i = 0; i < nsteps; i++)
        for (int q = 0; q < 3; q++) {
            float t = 0;
            cudaEventElapsedTime(&t, E.ev[4 * i + q], E.ev[4 * i + q + 1]);
            acc[q] += t;
        }
    sh.it_host += nsteps;
    for (int q = 0; q < 3; q++) ms[q] = (float)(acc[q] / nsteps);
    return BP_OK;
}

}  // extern "C"

namespace bpk {
// Algorithmic HBM bytes per updated cell of each phase: words touched once per
// phase per updated cell (each array element once; neighbour re-reads and the
// slab-only CPML variables not counted):
//   V: read stresses+p, read+write vu,vw, read coefficients
//   T: read vu,vw, read+write stresses+p, read coefficients
// An indexed medium reads one index byte per cell and phase in place of the
// coefficients (its table stays in L1).
void algorithmic_bpc(const bp_config& c, bool indexed, double bpc[2]) {
    double fb, cb;
    if (c.precision == BP_PREC_FP64) { fb = 8; cb = 8; }
    else if (c.precision == BP_PREC_FP32) { fb = 4; cb = 4; }
    else if (c.precision == BP_PREC_CBF16) { fb = 3; cb = 3; }
    else { fb = 3; cb = c.comp_coef_lo ? 3 : 2; }
    const int nvc = c.dim == 3 ? 10 : 7, ntc = c.dim == 3 ? 7 : 5;
    const double v_coef = indexed ? 1.0 : nvc * cb, t_coef = indexed ? 1.0 : ntc * cb;
    if (c.dim == 3) {
        bpc[0] = (7 + 2 * 6) * fb + v_coef;
        bpc[1] = (6 + 2 * 7) * fb + t_coef;
    } else {
        bpc[0] = (4 + 2 * 4) * fb + v_coef;
        bpc[1] = (4 + 2 * 4) * fb + t_coef;
    }
}
}  // namespace bpk

extern "C" {

int bp_algorithmic_bytes(bp_sim* s, double bpc[2], long long* cells) {
    if (!s || !bpc) { set_error("bad arguments"); return BP_ERR_ARG; }
    algorithmic_bpc(s->shot.cfg, s->shot.med_tuples > 0, bpc);
    if (cells) *cells = s->shot.cells;
    return BP_OK;
}

int bp_get_medium_tuples(bp_sim* s, int* ntuples) {
    if (!s || !ntuples) { set_error("bad arguments"); return BP_ERR_ARG; }
    *ntuples = s->shot.med_tuples;
    return BP_OK;
}

int bp_launches_per_step(bp_sim* s, int* n) {
    if (!s || !n) { set_error("bad arguments"); return BP_ERR_ARG; }
    *n = s->run.fused ? 1 : (s->run.inter ? (s->run.fused_post() ? 1 : 2) : s->run.launches_per_step());
    return BP_OK;
}

int bp_get_kernel(bp_sim* s, int* variant) {
    if (!s || !variant) { set_error("bad arguments"); return BP_ERR_ARG; }
    *variant = s->run.family();
    return BP_OK;
}

int bp_profile_fused(bp_sim* s, int nsteps, float* ms, double* bytes_per_cell) {
    if (!s || !ms || nsteps < 1) { set_error("bad arguments"); return BP_ERR_ARG; }
    Shot& sh = s->shot;
    Runner& R = s->run;
    if (sh.ntiles_f <= 0 || sh.cfg.rounding != BP_ROUND_FAST) {
        set_error("the fused step kernel does not apply to this simulation");
        return BP_ERR_ARG;
    }
    SIM_CK(cudaSetDevice(s->device));
    const int pairs = std::min((nsteps + 1) / 2, (sh.cfg.nt - sh.it_host) / 2);
    if (pairs < 1) { set_error("no steps left to profile"); return BP_ERR_STATE; }
    EventRing E;
    SIM_CK(E.make((size_t)3 * pairs));
    cudaError_t e = cudaSuccess;
    for (int i = 0; i < pairs && e == cudaSuccess; i++) {
        cudaEvent_t* ev = &E.ev[3 * i];
        cudaEventRecord(ev[0], s->st);
        e = launch_fused(R.prec, R.order, R.d_shots, R.nshots, R.ntiles_f, 0, 0, R.grid_f, s->st);
        cudaEventRecord(ev[1], s->st);
        if (e == cudaSuccess) e = launch_fused(R.prec, R.order, R.d_shots, R.nshots, R.ntiles_f, 1, 1, R.grid_f, s->st);
        cudaEventRecord(ev[2], s->st);
        if (e == cudaSuccess) e = launch_advance(R.d_shots, R.nshots, 2, s->st);
        R.launches += 3;
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(s->st);
    if (e != cudaSuccess) { set_error(cudaGetErrorString(e)); return BP_ERR_CUDA; }
    double acc = 0;
    for (int i = 0; i < pairs; i++) {
        float t0 = 0, t1 = 0;
        cudaEventElapsedTime(&t0, E.ev[3 * i], E.ev[3 * i + 1]);
        cudaEventElapsedTime(&t1, E.ev[3 * i + 1], E.ev[3 * i + 2]);
        acc += t0 + t1;
    }
    sh.it_host += 2 * pairs;
    *ms = (float)(acc / (2.0 * pairs));
    if (bytes_per_cell) {
        const bp_config& c = sh.cfg;
        const double fb = c.precision == BP_PREC_FP32 ? 4 : 3;
        const double cb = c.precision == BP_PREC_FP32 ? 4 : ((c.comp_coef_lo || c.precision == BP_PREC_CBF16) ? 3 : 2);
        // 2D: the 8 fields read and written once, 7 V + 5 T coefficients read
        // once (an indexed medium: one index byte)
        *bytes_per_cell = 2 * 8 * fb + (sh.med_tuples > 0 ? 1.0 : 12 * cb);
    }
    return BP_OK;
}

int bp_launch_count(bp_sim* s, long long* n) {
    if (!s || !n) { set_error("bad arguments"); return BP_ERR_ARG; }
    *n = s->run.launches;
    return BP_OK;
}

int bp_rel_l2_device(const float* d_x, const float* d_ref, size_t n, double* rel) {
    if (!d_x || !d_ref || !rel) { set_error("bad arguments"); return BP_ERR_ARG; }
    const int nb = reduce_blocks();
    double* scratch = nullptr;
    SIM_CK(cudaMalloc(&scratch, (2 * (size_t)nb + 2) * sizeof(double)));
    double h[2] = {0, 0};
    cudaError_t e = launch_rel_l2(d_x, d_ref, (long long)n, scratch, scratch + 2 * nb, 0);
    if (e == cudaSuccess) e = cudaMemcpy(h, scratch + 2 * nb, 2 * sizeof(double), cudaMemcpyDeviceToHost);
    cudaFree(scratch);
    if (e != cudaSuccess) { set_error(cudaGetErrorString(e)); return BP_ERR_CUDA; }
    *rel = h[1] > 0 ? std::sqrt(h[0] / h[1]) : std::sqrt(h[0]);
    return BP_OK;
}

int bp_trace_rel_l2(bp_sim* x, bp_sim* ref, int comp, double* rel) {
    if (!x || !ref || !rel || comp < 0 || comp >= BP_NTRACE) { set_error("bad arguments"); return BP_ERR_ARG; }
    if (x->shot.nurec != ref->shot.nurec || x->shot.cfg.nt != ref->shot.cfg.nt) { set_error("traces differ in shape"); return BP_ERR_ARG; }
    SIM_CK(cudaStreamSynchronize(x->st));
    SIM_CK(cudaStreamSynchronize(ref->st));
    const size_t n = (size_t)x->shot.nurec * x->shot.cfg.nt;
    return bp_rel_l2_device(x->shot.desc.traces + comp * n, ref->shot.desc.traces + comp * n, n, rel);
}

void bp_destroy(bp_sim* s) {
    if (!s) return;
    cudaSetDevice(s->device);
    if (s->st) cudaStreamSynchronize(s->st);
    s->run.reset_graph();
    s->shot.destroy();
    if (s->d_zf) arena_release(s->d_zf, s->d_zf_bytes);
    if (s->st) cudaStreamDestroy(s->st);
    delete s;
}

int bp_set_z_spacing(bp_sim* s, const double* dz, int n) {
    if (!s || !dz) { set_error("bad arguments"); return BP_ERR_ARG; }
    Shot& sh = s->shot;
    const bp_config& c = sh.cfg;
    if (c.precision != BP_PREC_FP32 || c.rounding != BP_ROUND_FAST || c.order != 2) {
        set_error("the variable z grid runs FP32 with fast rounding at order 2");
        return BP_ERR_ARG;
    }
    if (sh.it_host != 0 || s->d_zf) { set_error("set the z spacing once, before the first step"); return BP_ERR_STATE; }
    const int nzp = sh.desc.nz;
    if (n != nzp - 1) { set_error("dz needs nz + 2 npml - 1 spacings"); return BP_ERR_ARG; }
    const double H = (double)c.dx;
    double dmin = H;
    for (int k = 0; k < n; k++) {
        if (!(dz[k] > 0) || !std::isfinite(dz[k])) { set_error("spacings must be positive and finite"); return BP_ERR_ARG; }
        const bool cpml_row = k < c.npml + 1 || k >= n - (c.npml + 1);
        if (cpml_row && dz[k] != H) { set_error("the CPML rows keep the spacing dx"); return BP_ERR_ARG; }
        dmin = std::min(dmin, dz[k]);
    }
    if (s->cfl_dtmax > 0 && (double)c.dt > s->cfl_dtmax * (dmin / H)) {
        char buf[160];
        snprintf(buf, sizeof buf, "dt=%g exceeds the stability limit %g of the finest spacing %g", (double)c.dt,
                 s->cfl_dtmax * (dmin / H), dmin);
        set_error(buf);
        return BP_ERR_CFL;
    }
    // fwd[z] = 1/dz[z]; bwd[z] = 2/(dz[z-1] + dz[z]); rows without both
    // neighbours (never updated) take 1/dx
    std::vector<float> zf(2 * (size_t)nzp);
    for (int z = 0; z < nzp; z++) {
        zf[z] = (float)(z < n ? 1.0 / dz[z] : 1.0 / H);
        zf[nzp + z] = (float)((z >= 1 && z < n) ? 2.0 / (dz[z - 1] + dz[z]) : 1.0 / H);
    }
    SIM_CK(cudaSetDevice(s->device));
    SIM_CK(cudaStreamSynchronize(s->st));
    SIM_CK(arena_alloc(zf.size() * 4, (void**)&s->d_zf, &s->d_zf_bytes));
    SIM_CK(cudaMemcpy(s->d_zf, zf.data(), zf.size() * 4, cudaMemcpyHostToDevice));
    sh.desc.zf = s->d_zf;
    SIM_CK(cudaMemcpy((void*)sh.d_desc, &sh.desc, sizeof(ShotDesc), cudaMemcpyHostToDevice));
    s->run.graded = true;
    s->run.select_kernels();
    s->run.reset_graph();
    return BP_OK;
}

// ---- reference-format text output (Float/main.cu:1501-1516,1563-1588) ----
static int write_rows(const std::string& path, const float* data, int nr, int nc) {
    FILE* fp = fopen(path.c_str(), "wt");
    if (!fp) { set_error("cannot open " + path); return BP_ERR_ARG; }
    for (int i = 0; i < nr; i++) {
        for (int j = 0; j < nc; j++) {
            fprintf(fp, "%e ", data[(size_t)i * nc + j]);
            if ((j + 1) % nc == 0) fprintf(fp, "\n");
        }
        fprintf(fp, "\n");
    }
    fclose(fp);
    return BP_OK;
}

static int write_bin(const std::string& path, const float* data, int ndims, const int* dims) {
    BinHeader h;
    std::memset(&h, 0, sizeof h);
    std::memcpy(h.magic, kBinMagic, 8);
    h.version = 1;
    h.dtype = 0;
    h.ndims = ndims;
    size_t n = 1;
    for (int i = 0; i < ndims; i++) { h.dims[i] = dims[i]; n *= (size_t)dims[i]; }
    FILE* fp = fopen(path.c_str(), "wb");
    if (!fp) { set_error("cannot open " + path); return BP_ERR_ARG; }
    bool ok = fwrite(&h, sizeof h, 1, fp) == 1 && (n == 0 || fwrite(data, 4, n, fp) == n);
    ok = (fclose(fp) == 0) && ok;
    if (!ok) { set_error("short write to " + path); return BP_ERR_ARG; }
    return BP_OK;
}

int bp_write_binary_outputs(bp_sim* s, const char* dir) {
    if (!s || !dir) { set_error("bad arguments"); return BP_ERR_ARG; }
    mkdir(dir, 0755);
    Shot& sh = s->shot;
    const int nt = sh.cfg.nt, nr = sh.cfg.nrec;
    const std::string d(dir);
    std::vector<float> all((size_t)BP_NTRACE * nr * nt);
    for (int c = 0; c < BP_NTRACE; c++) {
        int rc = bp_get_traces(s, c, all.data() + (size_t)c * nr * nt, (size_t)nr * nt);
        if (rc) return rc;
    }
    const int tdims[3] = {BP_NTRACE, nr, nt};
    int rc = write_bin(d + "/traces.bin", all.data(), 3, tdims);
    if (rc) return rc;
    const int nx = sh.desc.nx, ny = sh.desc.ny, nz = sh.desc.nz;
    const bool vol = sh.cfg.dim == 3 && sh.cfg.snap_y < 0;
    std::vector<float> snap(sh.snap_n);
    for (int k = 0; k < (int)sh.snap_steps.size(); k++) {
        for (int f = 0; f < BP_NFIELDS; f++) {
            if (sh.snap_off[(size_t)k * BP_NFIELDS + f] < 0) continue;
            rc = bp_get_snapshot(s, k, f, snap.data(), snap.size());
            if (rc) return rc;
            const int d3[3] = {nz, ny, nx}, d2[2] = {nz, nx};
            rc = vol ? write_bin(d + "/" + kFieldNames[f] + std::to_string(sh.snap_steps[k]) + ".bin", snap.data(), 3, d3)
                     : write_bin(d + "/" + kFieldNames[f] + std::to_string(sh.snap_steps[k]) + ".bin", snap.data(), 2, d2);
            if (rc) return rc;
        }
    }
    return BP_OK;
}

int bp_write_reference_outputs(bp_sim* s, const char* dir) {
    if (!s || !dir) { set_error("bad arguments"); return BP_ERR_ARG; }
    mkdir(dir, 0755);
    Shot& sh = s->shot;
    const int nt = sh.cfg.nt, nr = sh.cfg.nrec;
    const std::string d(dir);
    const char* sis[BP_NTRACE] = {"sisx.dat", "sisz.dat", "sisvu.dat", "sisvw.dat", "sisp.dat"};
    std::vector<float> buf((size_t)nr * nt);
    for (int c = 0; c < BP_NTRACE; c++) {
        int rc = bp_get_traces(s, c, buf.data(), buf.size());
        if (rc) return rc;
        rc = write_rows(d + "/" + sis[c], buf.data(), nr, nt);
        if (rc) return rc;
    }
    const int nx = sh.desc.nx, ny = sh.desc.ny, nz = sh.desc.nz;
    const bool slice = sh.cfg.dim == 3 && sh.cfg.snap_y >= 0;
    std::vector<float> snap(sh.snap_n), sl((size_t)nx * nz);
    for (int k = 0; k < (int)sh.snap_steps.size(); k++) {
        for (int f = 0; f < BP_NFIELDS; f++) {
            if (sh.snap_off[(size_t)k * BP_NFIELDS + f] < 0) continue;
            int rc = bp_get_snapshot(s, k, f, snap.data(), snap.size());
            if (rc) return rc;
            const float* src = snap.data();
            if (!slice && sh.cfg.dim == 3) {   // full volume: write the y = NY/2 slice like wfile3d
                for (int z = 0; z < nz; z++)
                    for (int x = 0; x < nx; x++) sl[(size_t)z * nx + x] = snap[(size_t)x + (size_t)(ny / 2) * nx + (size_t)z * nx * ny];
                src = sl.data();
            }
            rc = write_rows(d + "/" + kFieldNames[f] + std::to_string(sh.snap_steps[k]) + ".dat", src, nz, nx);
            if (rc) return rc;
        }
    }
    // final txx (Float/main.cu:1166-1175,1190)
    std::vector<float> full((size_t)nx * ny * nz);
    int rc = bp_get_field(s, BP_F_TXX, full.data(), full.size());
    if (rc) return rc;
    int jy = sh.cfg.dim == 3 ? ny / 2 : 0;
    for (int z = 0; z < nz; z++)
        for (int x = 0; x < nx; x++) sl[(size_t)z * nx + x] = full[(size_t)x + (size_t)jy * nx + (size_t)z * nx * ny];
    return write_rows(d + "/txx.dat", sl.data(), nz, nx);
}

}  // extern "C"
