// shot.cu - allocation and FP64 precompute of one shot's device state.
//
// Replaces Float/main.cu:300-1040 (93 separate cudaMalloc + H2D copies of
// full-volume arrays) with one arena per shot holding:
//   fields (13 in 3D, 8 in 2D), V and T coefficient sets, 1-D CPML profile
//   tables, slab-only CPML memory variables, the source wavelet, receiver
//   indices, trace and snapshot buffers, reduction scratch and the device copy
//   of the shot descriptor.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "shot.h"

namespace bpk {

static thread_local std::string g_last_error;
void set_error(const std::string& msg) { g_last_error = msg; }
const char* last_error_cstr() { return g_last_error.c_str(); }

#define BP_CK(call)                                                                        \
    do {                                                                                   \
        cudaError_t e_ = (call);                                                           \
        if (e_ != cudaSuccess) {                                                           \
            set_error(std::string(#call) + ": " + cudaGetErrorString(e_));                 \
            return e_ == cudaErrorMemoryAllocation ? BP_ERR_OOM : BP_ERR_CUDA;             \
        }                                                                                  \
    } while (0)

static bool field_used(int dim, int f) {
    if (dim == 3) return true;
    return !(f == BP_F_VUY || f == BP_F_VWY || f == BP_F_TYY || f == BP_F_TXY || f == BP_F_TYZ);
}
static bool vcoef_used(int dim, int c) { return dim == 3 || !(c == VC_RHO_Y || c == VC_CC1_Y || c == VC_CC2_Y); }
static bool tcoef_used(int dim, int c) { return dim == 3 || !(c == TC_MUXY || c == TC_MUYZ); }

int validate_config(const bp_config* c) {
    if (!c) { set_error("null config"); return BP_ERR_ARG; }
    if (c->dim != 2 && c->dim != 3) { set_error("dim must be 2 or 3"); return BP_ERR_ARG; }
    if (c->order != 2 && c->order != 4) { set_error("order must be 2 or 4"); return BP_ERR_ARG; }
    if (c->precision < BP_PREC_FP32 || c->precision > BP_PREC_CBF16) { set_error("bad precision"); return BP_ERR_ARG; }
    if (c->rounding != BP_ROUND_FAST && c->rounding != BP_ROUND_REFERENCE) { set_error("bad rounding"); return BP_ERR_ARG; }
    if (c->medium != BP_MEDIUM_AUTO && c->medium != BP_MEDIUM_DENSE) { set_error("bad medium mode"); return BP_ERR_ARG; }
    if (c->rounding == BP_ROUND_REFERENCE && c->precision != BP_PREC_FP32) {
        set_error("reference rounding applies to FP32 only");
        return BP_ERR_ARG;
    }
    if (c->nx < 1 || c->nz < 1 || (c->dim == 3 && c->ny < 1) || c->npml < 0) { set_error("bad grid size"); return BP_ERR_ARG; }
    const int hw = c->order / 2;
    const int nx = c->nx + 2 * c->npml, nz = c->nz + 2 * c->npml, ny = c->dim == 3 ? c->ny + 2 * c->npml : 1;
    if (nx < 2 * hw + 1 || nz < 2 * hw + 1 || (c->dim == 3 && ny < 2 * hw + 1)) { set_error("grid smaller than the stencil"); return BP_ERR_ARG; }
    // the phase kernels address cells with 32-bit offsets: every array (row
    // pitch x ny x nz cells, the pitch rounded up to 32) holds < 2^31 elements
    if ((long long)((nx + 31) & ~31) * ny * nz >= (1LL << 31)) {
        set_error("grid too large: the padded grid (row pitch x ny x nz, pitch = nx + 2 npml rounded up to 32) "
                  "must hold fewer than 2^31 cells");
        return BP_ERR_ARG;
    }
    if (!(c->dx > 0) || !(c->dt > 0) || c->nt < 1) { set_error("dx, dt must be > 0 and nt >= 1"); return BP_ERR_ARG; }
    if (!(c->f0 > 0)) { set_error("f0 must be > 0"); return BP_ERR_ARG; }
    if (c->npml > 0 && (!(c->pml_v0 > 0) || !(c->pml_r > 0) || !(c->pml_r < 1))) { set_error("bad CPML parameters"); return BP_ERR_ARG; }
    if (c->src_mask) {
        if (c->src_x < 0 || c->src_x >= nx || c->src_z < 0 || c->src_z >= nz || (c->dim == 3 && (c->src_y < 0 || c->src_y >= ny))) {
            set_error("source outside the padded grid"); return BP_ERR_ARG;
        }
    }
    if (c->nrec < 0 || (c->nrec > 0 && (!c->rec_x || !c->rec_z || (c->dim == 3 && !c->rec_y)))) { set_error("bad receiver arrays"); return BP_ERR_ARG; }
    for (int r = 0; r < c->nrec; r++) {
        int y = c->dim == 3 ? c->rec_y[r] : 0;
        if (c->rec_x[r] < 0 || c->rec_x[r] >= nx || c->rec_z[r] < 0 || c->rec_z[r] >= nz || y < 0 || y >= ny) {
            set_error("receiver " + std::to_string(r) + " outside the padded grid"); return BP_ERR_ARG;
        }
    }
    if (c->nsnap < 0 || (c->nsnap > 0 && !c->snap_steps)) { set_error("bad snapshot list"); return BP_ERR_ARG; }
    for (int k = 0; k < c->nsnap; k++)
        if (c->snap_steps[k] < 0 || c->snap_steps[k] >= c->nt) { set_error("snapshot step outside [0, nt)"); return BP_ERR_ARG; }
    if (c->dim == 3 && c->nsnap > 0 && c->snap_y >= ny) { set_error("snap_y outside the grid"); return BP_ERR_ARG; }
    return BP_OK;
}

namespace {
struct Arena {
    size_t off = 0;
    size_t take(size_t bytes) {
        size_t o = off;
        off += (bytes + 255) & ~(size_t)255;
        return o;
    }
};

struct Plan {
    int nx, ny, nz, pitch;
    long long ncell;
    Slab slab[3];
    long long slab_cells[3];
    int ns;                       // memory-variable slots per axis per phase
    size_t fe, ce, re;            // field, coefficient, real element sizes
    bool lo_f, lo_c;
    int nurec;
    size_t snap_n;
    int ncapt;
    // offsets
    size_t o_f[BP_NFIELDS], o_flo[BP_NFIELDS], o_vc[VC_COUNT], o_vclo[VC_COUNT], o_tc[TC_COUNT], o_tclo[TC_COUNT];
    size_t o_prof[3][4], o_psiV[3], o_psiT[3];
    size_t o_fb[BP_NFIELDS], o_flob[BP_NFIELDS], o_psiVb[3];   // second copy (fused step kernel)
    bool fused;
    size_t o_tr, o_tr64, o_wav, o_dyn, o_rtab, o_rec, o_recrow, o_recxu, o_step, o_blowup, o_snap, o_scratch, o_out, o_desc;
    size_t o_midx, o_mtab, o_mtmp;            // indexed medium: cell indices, tuple table, build scratch
    size_t total;
    size_t staging;               // transient medium upload
};

Slab make_slab(int n, int np, float H, int axis_x) {
    int L = 0, R0 = n;
    for (int i = 0; i < n; i++) {
        bool l, r;
        host_pml_region(n, np, H, i, &l, &r);
        if (l) L = i + 1;
        if (r && i < R0) R0 = i;
    }
    Slab s;
    if (axis_x) {
        L = (L + 3) & ~3;
        R0 = R0 & ~3;
    }
    if (L >= R0) { L = n; R0 = n; }  // slabs meet: the whole axis carries memory variables
    s.lo = L;
    s.hi0 = R0;
    s.width = L + (n - R0);
    if (axis_x) s.width = (s.width + 3) & ~3;
    return s;
}

void make_plan(const bp_config* c, int nurec, Plan& p) {
    const int dim = c->dim;
    p.nx = c->nx + 2 * c->npml;
    p.ny = dim == 3 ? c->ny + 2 * c->npml : 1;
    p.nz = c->nz + 2 * c->npml;
    p.pitch = (p.nx + 31) & ~31;
    p.ncell = (long long)p.pitch * p.ny * p.nz;
    p.ns = dim == 3 ? 4 : 3;
    const int prec = c->precision;
    p.fe = prec == BP_PREC_FP64 ? 8 : (prec == BP_PREC_FP32 ? 4 : 2);
    p.ce = p.fe;
    p.re = prec == BP_PREC_FP64 ? 8 : 4;
    p.lo_f = prec == BP_PREC_COMP16 || prec == BP_PREC_CBF16;
    p.lo_c = (prec == BP_PREC_COMP16 && c->comp_coef_lo) || prec == BP_PREC_CBF16;
    p.nurec = nurec;
    int ns_ax[3] = {p.nx, p.ny, p.nz};
    for (int a = 0; a < 3; a++) {
        if (a == 1 && dim == 2) { p.slab[a] = Slab{0, 1, 0}; p.slab_cells[a] = 0; continue; }
        p.slab[a] = make_slab(ns_ax[a], c->npml, c->dx, a == 0);
    }
    p.slab_cells[0] = (long long)p.nz * p.ny * p.slab[0].width;
    if (dim == 3) p.slab_cells[1] = (long long)p.nz * p.slab[1].width * p.pitch;
    p.slab_cells[2] = (long long)p.slab[2].width * p.ny * p.pitch;
    p.snap_n = (dim == 3 && c->snap_y >= 0) ? (size_t)p.nx * p.nz : (size_t)p.nx * p.ny * p.nz;
    p.ncapt = 0;
    for (int k = 0; k < c->nsnap; k++) {
        unsigned m = c->snap_masks ? c->snap_masks[k] : c->snap_fields;
        for (int f = 0; f < BP_NFIELDS; f++)
            if ((m >> f & 1u) && field_used(dim, f)) p.ncapt++;
    }
    Arena A;
    p.fused = fused_supported(prec, dim) && c->rounding == BP_ROUND_FAST;
    for (int f = 0; f < BP_NFIELDS; f++) {
        p.o_f[f] = p.o_flo[f] = p.o_fb[f] = p.o_flob[f] = (size_t)-1;
        if (!field_used(dim, f)) continue;
        p.o_f[f] = A.take(p.ncell * p.fe);
        if (p.lo_f) p.o_flo[f] = A.take(p.ncell);
        if (p.fused) {
            p.o_fb[f] = A.take(p.ncell * p.fe);
            if (p.lo_f) p.o_flob[f] = A.take(p.ncell);
        }
    }
    for (int k = 0; k < VC_COUNT; k++) {
        p.o_vc[k] = p.o_vclo[k] = (size_t)-1;
        if (!vcoef_used(dim, k)) continue;
        p.o_vc[k] = A.take(p.ncell * p.ce);
        if (p.lo_c) p.o_vclo[k] = A.take(p.ncell);
    }
    for (int k = 0; k < TC_COUNT; k++) {
        p.o_tc[k] = p.o_tclo[k] = (size_t)-1;
        if (!tcoef_used(dim, k)) continue;
        p.o_tc[k] = A.take(p.ncell * p.ce);
        if (p.lo_c) p.o_tclo[k] = A.take(p.ncell);
    }
    for (int a = 0; a < 3; a++) {
        for (int q = 0; q < 4; q++) p.o_prof[a][q] = (size_t)-1;
        p.o_psiV[a] = p.o_psiT[a] = p.o_psiVb[a] = (size_t)-1;
        if (a == 1 && dim == 2) continue;
        for (int q = 0; q < 4; q++) p.o_prof[a][q] = A.take((size_t)ns_ax[a] * p.re);
        p.o_psiV[a] = A.take((size_t)2 * p.ns * p.slab_cells[a] * p.re);
        if (p.fused) p.o_psiVb[a] = A.take((size_t)2 * p.ns * p.slab_cells[a] * p.re);
        p.o_psiT[a] = A.take((size_t)2 * p.ns * p.slab_cells[a] * p.re);
    }
    const size_t tr = (size_t)BP_NTRACE * nurec * c->nt;
    p.o_tr = A.take(tr * 4 + 4);
    p.o_tr64 = prec == BP_PREC_FP64 ? A.take(tr * 8 + 8) : (size_t)-1;
    p.o_wav = A.take((size_t)c->nt * (prec == BP_PREC_FP64 ? 8 : 4));
    p.o_dyn = A.take((size_t)c->nt * 4);
    p.o_rtab = A.take((size_t)c->nt * 4);
    p.o_rec = A.take((size_t)nurec * 8 + 8);
    p.o_recrow = A.take(((size_t)p.ny * p.nz + 1) * 4);
    p.o_recxu = A.take((size_t)nurec * 8 + 8);
    p.o_step = A.take(4);
    p.o_blowup = A.take(4);
    p.o_snap = A.take((size_t)p.ncapt * p.snap_n * 4 + 4);
    const int nb = scan_kr_blocks() > reduce_blocks() ? scan_kr_blocks() : reduce_blocks();
    p.o_scratch = A.take((size_t)2 * nb * 8);
    p.o_out = A.take(4 * 8);
    p.o_desc = A.take(sizeof(ShotDesc));
    p.o_midx = p.o_mtab = p.o_mtmp = (size_t)-1;
    if (prec != BP_PREC_FP64 && c->medium == BP_MEDIUM_AUTO) {
        p.o_midx = A.take((size_t)p.ncell);
        p.o_mtab = A.take((size_t)kMedMaxTuples * kMedRow * sizeof(float4));
        p.o_mtmp = A.take(medium_scratch_bytes());
    }
    p.total = A.off;
    p.staging = (size_t)9 * c->nx * (dim == 3 ? c->ny : 1) * c->nz * 4;
}

// Reference Ricker wavelet (Float/main.cu:1050,1059): float time, double PI
// literal and exp, rounded to float.
float ricker_float(int it, float DT, float F0, float T0) {
    const double PI = 3.1415926535;
    float tt = it * DT;
    float a = tt - T0;
    return (float)(-(1 - 2 * PI * PI * F0 * F0 * a * a) * exp(-PI * PI * F0 * F0 * a * a));
}
double ricker_double(int it, double DT, double F0, double T0) {
    const double PI = 3.1415926535;
    double a = it * DT - T0;
    return -(1 - 2 * PI * PI * F0 * F0 * a * a) * exp(-PI * PI * F0 * F0 * a * a);
}
}  // namespace

int Shot::plan_bytes(const bp_config* c, size_t* bytes) {
    int rc = validate_config(c);
    if (rc) return rc;
    Plan p;
    make_plan(c, c->nrec, p);   // upper bound: every receiver unique
    *bytes = p.total + p.staging;
    return BP_OK;
}

int Shot::create(const bp_config* c, const bp_medium* med, cudaStream_t st) {
    int rc = validate_config(c);
    if (rc) return rc;
    if (!med || !med->rho || !med->rhof || !med->M || !med->C || !med->H || !med->H2mu || !med->mu || !med->C1 || !med->C2) {
        set_error("medium arrays missing");
        return BP_ERR_ARG;
    }
    cfg = *c;
    const int dim = c->dim;
    const int nxp = c->nx + 2 * c->npml, nyp = dim == 3 ? c->ny + 2 * c->npml : 1;
    // copy caller arrays so the config stays valid after the call
    rec_x.assign(c->rec_x, c->rec_x + c->nrec);
    rec_z.assign(c->rec_z, c->rec_z + c->nrec);
    rec_y.assign(c->nrec, 0);
    if (dim == 3) rec_y.assign(c->rec_y, c->rec_y + c->nrec);
    snap_steps.assign(c->snap_steps, c->snap_steps + c->nsnap);
    snap_masks.resize(c->nsnap);
    for (int k = 0; k < c->nsnap; k++) snap_masks[k] = c->snap_masks ? c->snap_masks[k] : c->snap_fields;
    cfg.rec_x = rec_x.data(); cfg.rec_y = rec_y.data(); cfg.rec_z = rec_z.data();
    cfg.snap_steps = snap_steps.data(); cfg.snap_masks = snap_masks.data();

    // unique receiver cells (duplicates share one recorded trace)
    const long long pitch = (nxp + 31) & ~31;
    std::vector<long long> uidx;
    std::map<long long, int> seen;
    urec_of.resize(c->nrec);
    for (int r = 0; r < c->nrec; r++) {
        long long i = rec_x[r] + (long long)rec_y[r] * pitch + (long long)rec_z[r] * pitch * nyp;
        auto itf = seen.find(i);
        if (itf == seen.end()) { seen[i] = (int)uidx.size(); urec_of[r] = (int)uidx.size(); uidx.push_back(i); }
        else urec_of[r] = itf->second;
    }
    nurec = (int)uidx.size();

    Plan p;
    make_plan(&cfg, nurec, p);
    arena_bytes = p.total;
    BP_CK(arena_alloc(arena_bytes, &arena, &arena_alloc_bytes));
    BP_CK(cudaMemsetAsync(arena, 0, arena_bytes, st));
    char* A = static_cast<char*>(arena);
    auto at = [&](size_t o) -> void* { return o == (size_t)-1 ? nullptr : (void*)(A + o); };

    ShotDesc& S = desc;
    std::memset(&S, 0, sizeof(S));
    S.dim = dim; S.order = c->order; S.hw = c->order / 2;
    S.nx = p.nx; S.ny = p.ny; S.nz = p.nz; S.pitch = p.pitch;
    S.plane = (long long)p.pitch * p.ny;
    S.nseg = (p.nx + seg_cells() - 1) / seg_cells();
    S.nrows = p.ny * p.nz;
    S.tile0 = 0;
    S.tile0s = 0;
    S.nseg_s = (p.nx + staged_tile_width() - 1) / staged_tile_width();
    S.tile0m = 0;
    S.ncol_m = (p.nx + march_cells() - 1) / march_cells();
    S.tile0f = 0;
    S.ncol_f = fused_cols(p.nx);
    {
        int dev = 0, sms = 148;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        S.zseg_m = march_zseg(S.ncol_m, p.nz - 2 * S.hw, sms);
        S.zseg_f = fused_zseg(S.ncol_f, p.nz - 2 * S.hw, sms);
        S.nzs_f = (p.nz - 2 * S.hw + S.zseg_f - 1) / S.zseg_f;
    }
    S.nt = c->nt;
    S.dt = c->dt; S.dtd = c->dt; S.h = c->dx; S.hd = c->dx; S.inv_h = 1.0f / c->dx;
    for (int f = 0; f < BP_NFIELDS; f++) {
        S.f[f] = at(p.o_f[f]);
        S.flo[f] = (int8_t*)at(p.o_flo[f]);
        S.fb[f] = at(p.o_fb[f]);
        S.flob[f] = (int8_t*)at(p.o_flob[f]);
    }
    for (int k = 0; k < VC_COUNT; k++) { S.vc[k] = at(p.o_vc[k]); S.vclo[k] = (int8_t*)at(p.o_vclo[k]); }
    for (int k = 0; k < TC_COUNT; k++) { S.tc[k] = at(p.o_tc[k]); S.tclo[k] = (int8_t*)at(p.o_tclo[k]); }
    for (int a = 0; a < 3; a++) {
        S.pb[a] = at(p.o_prof[a][0]); S.pe[a] = at(p.o_prof[a][1]);
        S.pb2[a] = at(p.o_prof[a][2]); S.pe2[a] = at(p.o_prof[a][3]);
        S.slab[a] = p.slab[a];
        S.slab_cells[a] = p.slab_cells[a];
        S.psiV[a] = at(p.o_psiV[a]);
        S.psiVb[a] = at(p.o_psiVb[a]);
        S.psiT[a] = at(p.o_psiT[a]);
    }
    S.traces = (float*)at(p.o_tr);
    S.traces64 = (double*)at(p.o_tr64);
    S.wavelet = at(p.o_wav);
    S.dyn = (const float*)at(p.o_dyn);
    S.rtab = (const float*)at(p.o_rtab);
    S.rec_idx = (const long long*)at(p.o_rec);
    S.nrec = nurec;
    S.rec_row = (const int*)at(p.o_recrow);
    S.rec_xu = (const int2*)at(p.o_recxu);
    S.step_base = (int*)at(p.o_step);
    S.blowup = (int*)at(p.o_blowup);
    S.src_mask = c->src_mask;
    S.src_idx_valid = c->src_mask != 0;
    S.src_idx = c->src_x + (long long)(dim == 3 ? c->src_y : 0) * pitch + (long long)c->src_z * pitch * nyp;
    S.src_rec = -1;
    for (int u = 0; u < nurec; u++)
        if (S.src_idx_valid && uidx[u] == S.src_idx) { S.src_rec = u; break; }
    d_snap = (float*)at(p.o_snap);
    snap_n = p.snap_n;
    d_scratch = (double*)at(p.o_scratch);
    d_out = (double*)at(p.o_out);
    snap_off.assign((size_t)c->nsnap * BP_NFIELDS, -1);
    long long so = 0;
    for (int k = 0; k < c->nsnap; k++)
        for (int f = 0; f < BP_NFIELDS; f++)
            if ((snap_masks[k] >> f & 1u) && field_used(dim, f)) { snap_off[(size_t)k * BP_NFIELDS + f] = so; so += (long long)snap_n; }

    // ---- medium upload (transient) ----
    const size_t pn = (size_t)c->nx * (dim == 3 ? c->ny : 1) * c->nz;
    // the staging block comes from the arena cache, like the arena itself, so
    // a create after a destroy of similar size allocates nothing
    float* stage = nullptr;
    size_t stage_bytes = 0;
    BP_CK(arena_alloc(9 * pn * sizeof(float), (void**)&stage, &stage_bytes));
    const float* src9[9] = {med->rho, med->rhof, med->M, med->C, med->H, med->H2mu, med->mu, med->C1, med->C2};
    const float* dm[9];
    int rc2 = BP_OK;
    for (int k = 0; k < 9 && rc2 == BP_OK; k++) {
        dm[k] = stage + k * pn;
        cudaError_t e = cudaMemcpyAsync((void*)dm[k], src9[k], pn * sizeof(float), cudaMemcpyHostToDevice, st);
        if (e != cudaSuccess) { set_error(std::string("medium upload: ") + cudaGetErrorString(e)); rc2 = BP_ERR_CUDA; }
    }
    auto fail = [&](int code) { cudaStreamSynchronize(st); arena_release(stage, stage_bytes); return code; };
    if (rc2) return fail(rc2);

    // ---- CPML profiles, FP64 ----
    const int next[3] = {p.nx, p.ny, p.nz};
    for (int a = 0; a < 3; a++) {
        if (a == 1 && dim == 2) continue;
        cudaError_t e = launch_profile(c->precision, next[a], c->npml, c->dx, (double)c->dt, (double)c->pml_v0,
                                       (double)c->pml_r, (void*)S.pb[a], (void*)S.pe[a], (void*)S.pb2[a],
                                       (void*)S.pe2[a], st);
        if (e != cudaSuccess) { set_error(std::string("profile kernel: ") + cudaGetErrorString(e)); return fail(BP_ERR_CUDA); }
    }
    // ---- COMP16 exponent scan (Half/main.cu:745-809) ----
    em = 0; es = 0;
    if (c->precision == BP_PREC_COMP16) {
        cudaError_t e = launch_scan_kr(dim, p.nx, p.ny, p.nz, dm, c->nx, dim == 3 ? c->ny : 1, c->nz, c->npml,
                                       d_scratch, d_out, st);
        double kr[2] = {0, 0};
        if (e == cudaSuccess) e = cudaMemcpyAsync(kr, d_out, 2 * sizeof(double), cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) { set_error(std::string("exponent scan: ") + cudaGetErrorString(e)); return fail(BP_ERR_CUDA); }
        kmax = kr[0]; rmax = kr[1];
        float Kmax = (float)kmax, Rmax = (float)rmax, DT = c->dt;
        em = -23;
        if (Kmax > 0.0f && Rmax > 0.0f) {
            float er = 1.0f / sqrtf(DT * DT * Kmax * Rmax);
            em = (int)lrintf(-log2f(er * DT * Kmax));
        }
        es = 0;
    }
    // ---- staggered coefficients, FP64 ----
    {
        cudaError_t e = launch_coefs(c->precision, S, dm, c->nx, dim == 3 ? c->ny : 1, c->nz, c->npml, (double)c->dt, em, st);
        if (e != cudaSuccess) { set_error(std::string("coefficient kernel: ") + cudaGetErrorString(e)); return fail(BP_ERR_CUDA); }
    }
    // ---- indexed medium (at most 256 distinct coefficient tuples) ----
    S.med_idx = nullptr;
    S.ctab = nullptr;
    S.med_tuples = 0;
    med_tuples = 0;
    if (p.o_midx != (size_t)-1) {
        uint8_t* midx = (uint8_t*)at(p.o_midx);
        float4* mtab = (float4*)at(p.o_mtab);
        int n = 0;
        cudaError_t e = build_medium_index(c->precision, S, midx, mtab, at(p.o_mtmp), (size_t)p.ncell, &n, st);
        if (e != cudaSuccess) { set_error(std::string("medium index: ") + cudaGetErrorString(e)); return fail(BP_ERR_CUDA); }
        if (n > 0) {
            S.med_idx = midx;
            S.ctab = mtab;
            S.med_tuples = n;
            med_tuples = n;
        }
    }
    // ---- wavelet, dynamic scale, receivers ----
    std::vector<float> wf(c->nt);
    std::vector<double> wd;
    const float T0 = c->t0 > 0 ? c->t0 : (float)(1.2 / c->f0);
    const double T0d = c->t0 > 0 ? (double)c->t0 : 1.2 / (double)c->f0;
    if (c->precision == BP_PREC_FP64) {
        wd.resize(c->nt);
        for (int it = 0; it < c->nt; it++) wd[it] = ricker_double(it, c->dt, c->f0, T0d);
    } else {
        for (int it = 0; it < c->nt; it++) wf[it] = ricker_float(it, c->dt, c->f0, T0);
    }
    dyn.assign(c->nt, 1.0f);
    std::vector<float> rtab(c->nt, 1.0f);
    if (c->precision == BP_PREC_COMP16) {
        // S.out_* and inj_scale: 2^-es, 2^(em-es), 2^es (Half/main.cu:802-806)
        S.out_stress = ldexpf(1.0f, -es);
        S.out_vel = ldexpf(1.0f, em - es);
        S.inj_scale = ldexpf(1.0f, es);
        if (c->dyn_scale) {
            // Half/main.cu:116-122,1326-1364: every 100 steps the scale moves to
            // 1 + 15 it/(NT-1); the whole state is multiplied by target/current.
            float cur = 1.0f;
            for (int it = 0; it < c->nt; it++) {
                if (it == 0 || it % 100 == 0) {
                    float target = c->nt <= 1 ? 16.0f : 1.0f + (16.0f - 1.0f) * ((float)it / (float)(c->nt - 1));
                    float ratio = target / cur;
                    if (fabsf(ratio - 1.0f) > 1.0e-6f) { rtab[it] = ratio; cur = target; }
                }
                dyn[it] = cur;
            }
        }
    }
    // host staging for the small uploads must outlive the async copies: sync below
    cudaError_t e = cudaSuccess;
    if (c->precision == BP_PREC_FP64) e = cudaMemcpyAsync((void*)S.wavelet, wd.data(), c->nt * 8, cudaMemcpyHostToDevice, st);
    else e = cudaMemcpyAsync((void*)S.wavelet, wf.data(), c->nt * 4, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync((void*)S.dyn, dyn.data(), c->nt * 4, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync((void*)S.rtab, rtab.data(), c->nt * 4, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess && nurec > 0)
        e = cudaMemcpyAsync((void*)S.rec_idx, uidx.data(), nurec * sizeof(long long), cudaMemcpyHostToDevice, st);
    // receivers by row (row key z * ny + y), sorted by x, for the T phase that
    // records them; it may do so only if every receiver and the source lie in
    // cells it visits (the chunk of x, and rows y, z, inside the stencil border)
    const int hwd = S.hw;
    auto visited = [&](long long i) {
        const int x = (int)(i % p.pitch), y = (int)((i / p.pitch) % p.ny), z = (int)(i / S.plane);
        const int x0 = x & ~3;
        return z >= hwd && z < p.nz - hwd && (dim == 2 || (y >= hwd && y < p.ny - hwd)) && x0 < p.nx - hwd &&
               x0 + 3 >= hwd;
    };
    std::vector<int> row_start((size_t)p.ny * p.nz + 1, 0);
    std::vector<std::pair<long long, int>> byrow(nurec);   // (row key * pitch + x, unique index)
    post_in_t = !S.src_idx_valid || visited(S.src_idx);
    for (int u = 0; u < nurec; u++) {
        const long long i = uidx[u];
        post_in_t = post_in_t && visited(i);
        byrow[u] = {i, u};                  // i = key * pitch + x orders by (row key, x)
    }
    std::sort(byrow.begin(), byrow.end());
    std::vector<int2> xu(nurec);
    for (int q = 0; q < nurec; q++) {
        const long long key = byrow[q].first / p.pitch;
        row_start[key + 1]++;
        xu[q] = make_int2((int)(byrow[q].first % p.pitch), byrow[q].second);
    }
    for (size_t k = 1; k < row_start.size(); k++) row_start[k] += row_start[k - 1];
    // with many receivers the chunks that hold them carry all the recording
    // while k_post spreads it over its own grid: measured on B200, 2000
    // receivers (4040 x 2040) are 1.2 % faster per step recorded in the T phase,
    // 65,536 (a 256 x 256 surface array on 552 x 552 x 424) 2.7 % slower
    // the fused step kernel records and injects in its stress phase only, so it
    // needs every receiver and the source in cells that phase visits
    const bool rec_in_t = post_in_t;
    post_in_t = post_in_t && nurec <= 8192;
    if (e == cudaSuccess)
        e = cudaMemcpyAsync((void*)S.rec_row, row_start.data(), row_start.size() * 4, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess && nurec > 0)
        e = cudaMemcpyAsync((void*)S.rec_xu, xu.data(), (size_t)nurec * 8, cudaMemcpyHostToDevice, st);
    ntiles = apply_tile_shape(S, dim, c->precision, default_tile_shape(dim, c->precision));
    {
        int dev = 0, sms = 148;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        S.item0_i = 0;
        S.band0_i = 0;
        nitems_i = apply_bands(S, dim, ntiles, inter_occupancy(c->precision, dim, c->order, c->rounding) * sms);
    }
    d_desc = (ShotDesc*)(A + p.o_desc);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(d_desc, &S, sizeof(ShotDesc), cudaMemcpyHostToDevice, st);
    // the first source sample, injected before the first V phase (Float/main.cu:1055-1062)
    if (e == cudaSuccess) e = launch_inject(c->precision, d_desc, 1, 0, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    arena_release(stage, stage_bytes);
    if (e != cudaSuccess) { set_error(std::string("shot set-up: ") + cudaGetErrorString(e)); return BP_ERR_CUDA; }

    long long cx = p.nx - 2 * S.hw, cz = p.nz - 2 * S.hw, cy = dim == 3 ? p.ny - 2 * S.hw : 1;
    cells = cx * cy * cz;
    ntiles_s = (long long)S.nseg_s * ((S.nrows + staged_tile_rows() - 1) / staged_tile_rows());
    ntiles_m = dim == 2 ? (long long)S.ncol_m * ((p.nz - 2 * S.hw + S.zseg_m - 1) / S.zseg_m) : 0;
    ntiles_f = p.fused && rec_in_t ? (long long)S.ncol_f * S.nzs_f : 0;
    it_host = 0;
    return BP_OK;
}

std::vector<std::pair<void*, size_t>> Shot::state_regions() const {
    std::vector<std::pair<void*, size_t>> r;
    const int dim = cfg.dim, prec = cfg.precision;
    const size_t ncell = (size_t)desc.pitch * desc.ny * desc.nz;
    const size_t fe = prec == BP_PREC_FP64 ? 8 : (prec == BP_PREC_FP32 ? 4 : 2);
    const size_t re = prec == BP_PREC_FP64 ? 8 : 4;
    const size_t ns = dim == 3 ? 4 : 3;
    for (int f = 0; f < BP_NFIELDS; f++) {
        if (!field_used(dim, f)) continue;
        r.emplace_back(desc.f[f], ncell * fe);
        if (prec == BP_PREC_COMP16 || prec == BP_PREC_CBF16) r.emplace_back(desc.flo[f], ncell);
    }
    for (int a = 0; a < 3; a++) {
        if (!desc.psiV[a]) continue;
        r.emplace_back(desc.psiV[a], 2 * ns * (size_t)desc.slab_cells[a] * re);
        r.emplace_back(desc.psiT[a], 2 * ns * (size_t)desc.slab_cells[a] * re);
    }
    const size_t tr = (size_t)BP_NTRACE * nurec * cfg.nt;
    r.emplace_back(desc.traces, tr * 4);
    if (desc.traces64) r.emplace_back(desc.traces64, tr * 8);
    size_t ncapt = 0;
    for (long long o : snap_off) ncapt += o >= 0;
    if (ncapt) r.emplace_back(d_snap, ncapt * snap_n * 4);
    return r;
}

// ---- arena cache --------------------------------------------------------
// A destroyed shot's arena is kept for the next shot of a similar size on the
// same device instead of being returned with cudaFree, whose cost for a GB-size
// block (0.4-1 s measured on B200) would dominate short runs and the
// create/destroy churn of the serving loop.  Bounded per device (a quarter of
// its memory, at most 32 GiB; BP_ARENA_CACHE_MB overrides, 0 disables);
// emptied when an allocation fails, and by bp_release_cached_memory.
namespace {
struct CachedArena {
    int device;
    void* ptr;
    size_t bytes;
};
std::mutex g_arena_mu;
std::vector<CachedArena> g_arenas;

size_t arena_cache_limit(int device) {
    static long long env = -2;
    if (env == -2) {
        const char* v = getenv("BP_ARENA_CACHE_MB");
        env = v ? atoll(v) : -1;
    }
    if (env >= 0) return (size_t)env << 20;
    // the device's total memory, queried once per device (cudaMemGetInfo took
    // tens of ms in some calls, and this runs on every release)
    static std::mutex mu;
    static std::map<int, size_t> limits;
    std::lock_guard<std::mutex> g(mu);
    auto it = limits.find(device);
    if (it != limits.end()) return it->second;
    size_t total = 0, freeb = 0;
    int cur = -1;
    cudaGetDevice(&cur);
    if (cur != device) return 0;
    if (cudaMemGetInfo(&freeb, &total) != cudaSuccess) { cudaGetLastError(); return 0; }
    return limits[device] = std::min(total / 4, (size_t)32 << 30);
}

void free_cached(int device) {   // g_arena_mu held; device -1 = all devices
    int cur = -1;
    cudaGetDevice(&cur);
    for (size_t i = 0; i < g_arenas.size();) {
        if (device < 0 || g_arenas[i].device == device) {
            if (g_arenas[i].device != cur) cudaSetDevice(g_arenas[i].device);
            cudaFree(g_arenas[i].ptr);
            g_arenas.erase(g_arenas.begin() + i);
        } else {
            i++;
        }
    }
    if (cur >= 0) cudaSetDevice(cur);
}
}  // namespace

// An arena of at least `bytes` on the current device: a cached one of up to
// 1.25x that size, else a new allocation (after emptying this device's cache
// if the first attempt fails).  *got is the block's real size.
// Injected allocation failure (bp_debug_fail_allocation): the number of
// arena requests left until the one that fails, 0 = none armed.
static std::atomic<long long> g_fail_in{0};

void arm_allocation_failure(long long nth) { g_fail_in.store(nth > 0 ? nth : 0); }

cudaError_t arena_alloc(size_t bytes, void** ptr, size_t* got) {
    // a request the test hook marks fails like an exhausted device, before it
    // takes a cached block or calls cudaMalloc, so nothing is held
    for (long long n = g_fail_in.load(); n > 0;) {
        if (g_fail_in.compare_exchange_weak(n, n - 1)) {
            if (n == 1) return cudaErrorMemoryAllocation;
            break;
        }
    }
    int dev = 0;
    cudaGetDevice(&dev);
    {
        std::lock_guard<std::mutex> g(g_arena_mu);
        int best = -1;
        for (int i = 0; i < (int)g_arenas.size(); i++) {
            const CachedArena& a = g_arenas[i];
            if (a.device == dev && a.bytes >= bytes && a.bytes <= bytes + bytes / 4 &&
                (best < 0 || a.bytes < g_arenas[best].bytes))
                best = i;
        }
        if (best >= 0) {
            *ptr = g_arenas[best].ptr;
            *got = g_arenas[best].bytes;
            g_arenas.erase(g_arenas.begin() + best);
            return cudaSuccess;
        }
    }
    cudaError_t e = cudaMalloc(ptr, bytes);
    if (e == cudaErrorMemoryAllocation) {
        cudaGetLastError();
        {
            std::lock_guard<std::mutex> g(g_arena_mu);
            free_cached(dev);
        }
        e = cudaMalloc(ptr, bytes);
    }
    if (e == cudaSuccess) *got = bytes;
    return e;
}

void arena_release(void* ptr, size_t bytes) {
    if (!ptr) return;
    int dev = 0;
    cudaGetDevice(&dev);
    const size_t limit = arena_cache_limit(dev);
    std::lock_guard<std::mutex> g(g_arena_mu);
    size_t held = 0;
    for (const CachedArena& a : g_arenas)
        if (a.device == dev) held += a.bytes;
    // evict the oldest entries of this device until the block fits
    for (size_t i = 0; held + bytes > limit && i < g_arenas.size();) {
        if (g_arenas[i].device == dev) {
            held -= g_arenas[i].bytes;
            cudaFree(g_arenas[i].ptr);
            g_arenas.erase(g_arenas.begin() + i);
        } else {
            i++;
        }
    }
    if (held + bytes <= limit) g_arenas.push_back({dev, ptr, bytes});
    else cudaFree(ptr);
}

void release_cached_arenas(int device) {
    std::lock_guard<std::mutex> g(g_arena_mu);
    free_cached(device);
}

int Shot::blowup_step(cudaStream_t st) const {
    int h = 0;
    if (!desc.blowup) return 0;
    if (cudaMemcpyAsync(&h, desc.blowup, sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
        return 0;
    return h;
}

cudaError_t Shot::copy_traces(int comp, float* host) const {
    const size_t nt = cfg.nt, nr = cfg.nrec;
    const float* src = desc.traces + (size_t)comp * nurec * nt;
    // receivers all distinct and in order (the usual case): one copy straight
    // into the caller's buffer, at full speed when that buffer is pinned
    bool identity = (size_t)nurec == nr;
    for (size_t r = 0; identity && r < nr; r++) identity = (size_t)urec_of[r] == r;
    if (identity) return nr ? cudaMemcpy(host, src, nr * nt * 4, cudaMemcpyDeviceToHost) : cudaSuccess;
    // receivers sharing a cell: the unique traces, then one row per receiver
    std::vector<float> u((size_t)nurec * nt);
    if (!u.empty()) {
        const cudaError_t e = cudaMemcpy(u.data(), src, u.size() * 4, cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) return e;
    }
    for (size_t r = 0; r < nr; r++) std::memcpy(host + r * nt, u.data() + (size_t)urec_of[r] * nt, nt * 4);
    return cudaSuccess;
}

void Shot::destroy() {
    if (arena) arena_release(arena, arena_alloc_bytes);
    arena = nullptr;
}

}  // namespace bpk
