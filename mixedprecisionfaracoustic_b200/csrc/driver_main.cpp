// driver_main.cpp - drop-in for the reference program's main()
// (Float/main.cu:300-1477 and Half/main.cu:376-1852).
//
//   biot_reference_run [--precision fp32|comp16|cbf16|fp64] [--nt N] [--out DIR]
//                      [--n NX NY NZ] [--np NP] [--rounding reference|fast]
//
// FP32 runs round like the reference's Float build (BP_ROUND_REFERENCE) unless
// --rounding fast: the outputs then match the reference program's own to the
// last digits its text format keeps.
//
// Same model (create_model: borehole in a porous formation), same grid
// (128^3 + 2*32 CPML, H = 0.01 m, DT = 0.9 us), same Ricker source (F0 = 3 kHz
// on txx, tyy, tzz at (NX/2, NY/2, 20+NP)), same vertical receiver line and
// snapshots, and the same 16 text files, written through the C ABI.
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "biot.h"

static int die(int rc, const char* what) {
    fprintf(stderr, "%s failed: %s (%s)\n", what, bp_error_string(rc), bp_last_error());
    return 1;
}

int main(int argc, char** argv) {
    int prec = BP_PREC_FP32, NT = 3500, NX = 128, NY = 128, NZ = 128, NP = 32, rounding = -1;
    std::string out = ".";
    for (int i = 1; i < argc; i++) {
        std::string a = argv[i];
        if (a == "--precision" && i + 1 < argc) {
            std::string p = argv[++i];
            prec = p == "comp16" ? BP_PREC_COMP16 : (p == "fp64" ? BP_PREC_FP64 : (p == "cbf16" ? BP_PREC_CBF16 : BP_PREC_FP32));
        } else if (a == "--nt" && i + 1 < argc) NT = atoi(argv[++i]);
        else if (a == "--out" && i + 1 < argc) out = argv[++i];
        else if (a == "--np" && i + 1 < argc) NP = atoi(argv[++i]);
        else if (a == "--rounding" && i + 1 < argc) rounding = std::string(argv[++i]) == "fast" ? BP_ROUND_FAST : BP_ROUND_REFERENCE;
        else if (a == "--n" && i + 3 < argc) { NX = atoi(argv[++i]); NY = atoi(argv[++i]); NZ = atoi(argv[++i]); }
        else { fprintf(stderr, "usage: %s [--precision fp32|comp16|cbf16|fp64] [--nt N] [--out DIR] [--n NX NY NZ] [--np NP] [--rounding reference|fast]\n", argv[0]); return 2; }
    }
    auto t0 = std::chrono::steady_clock::now();
    const int NXe = NX + 2 * NP, NYe = NY + 2 * NP, NZe = NZ + 2 * NP;
    const size_t n = (size_t)NX * NY * NZ;
    std::vector<float> med(9 * n);
    int rc = bp_medium_reference_borehole(NX, NY, NZ, med.data());
    if (rc) return die(rc, "bp_medium_reference_borehole");
    bp_medium m{med.data(), med.data() + n, med.data() + 2 * n, med.data() + 3 * n, med.data() + 4 * n,
                med.data() + 5 * n, med.data() + 6 * n, med.data() + 7 * n, med.data() + 8 * n};
    // receivers: the vertical line through the source column (Float/main.cu:1085-1093)
    const int sx = NXe / 2, sy = NYe / 2, sz = 20 + NP;
    std::vector<int> rx(NZe, sx), ry(NZe, sy), rz(NZe);
    for (int iz = 0; iz < NZe; iz++) rz[iz] = iz;
    // snapshots (Float/main.cu:1094-1163): 500 -> txx vux vwx vuz vwz; 1000..3000 -> txx
    std::vector<int> ss;
    std::vector<unsigned> sm;
    const unsigned F500 = (1u << BP_F_TXX) | (1u << BP_F_VUX) | (1u << BP_F_VWX) | (1u << BP_F_VUZ) | (1u << BP_F_VWZ);
    for (int s = 500; s <= 3000; s += 500)
        if (s < NT) { ss.push_back(s); sm.push_back(s == 500 ? F500 : (1u << BP_F_TXX)); }
    bp_config c;
    memset(&c, 0, sizeof c);
    c.dim = 3; c.nx = NX; c.ny = NY; c.nz = NZ; c.npml = NP; c.order = 2; c.precision = prec; c.nt = NT;
    c.dx = 0.01f;                       // float H = 0.01
    c.dt = (float)(0.9 * pow(10.0, -6)); // float DT = 0.9 * pow(10.0, -6)
    c.f0 = (float)(3 * pow(10.0, 3));
    c.t0 = (float)(1.2 / c.f0);
    c.pml_v0 = 4000.0f;
    c.pml_r = (float)(1.0 * pow(10.0, -6));
    c.src_x = sx; c.src_y = sy; c.src_z = sz; c.src_mask = BP_SRC_TAU;
    c.nrec = NZe; c.rec_x = rx.data(); c.rec_y = ry.data(); c.rec_z = rz.data();
    c.nsnap = (int)ss.size(); c.snap_steps = ss.data(); c.snap_masks = sm.data(); c.snap_y = NYe / 2;
    c.device = 0; c.comp_coef_lo = 1; c.dyn_scale = 1; c.check_cfl = 0;
    c.rounding = prec == BP_PREC_FP32 ? (rounding < 0 ? BP_ROUND_REFERENCE : rounding) : BP_ROUND_FAST;
    bp_sim* sim = nullptr;
    rc = bp_create(&c, &m, &sim);
    if (rc) return die(rc, "bp_create");
    auto t1 = std::chrono::steady_clock::now();
    for (int it = 0; it < NT; it += 100) {
        printf("it=%d\n", it);
        rc = bp_run(sim, NT - it < 100 ? NT - it : 100);
        if (rc) return die(rc, "bp_run");
    }
    rc = bp_sync(sim);
    if (rc) return die(rc, "bp_sync");
    auto t2 = std::chrono::steady_clock::now();
    rc = bp_write_reference_outputs(sim, out.c_str());
    if (rc) return die(rc, "bp_write_reference_outputs");
    auto t3 = std::chrono::steady_clock::now();
    double loop = std::chrono::duration<double>(t2 - t1).count();
    printf("NZ_ext = %d NY_ext = %d NX_ext = %d\n", NZe, NYe, NXe);
    printf("setup %.3f s, time loop %.3f s (%.1f Mcell-updates/s), output %.3f s\n",
           std::chrono::duration<double>(t1 - t0).count(), loop,
           (double)(NXe - 2) * (NYe - 2) * (NZe - 2) * NT / loop / 1e6, std::chrono::duration<double>(t3 - t2).count());
    bp_destroy(sim);
    return 0;
}
