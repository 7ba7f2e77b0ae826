// medium.cpp - host-side medium builders and the stability limit.
//
// bp_medium_reference_borehole restates the reference's create_model
// (Float/main.cu:1590-1655) with its exact float/double promotions, so the
// drop-in run sees the same cell-centred Biot coefficients as the reference.
#include <algorithm>
#include <cmath>
#include <cstddef>
#include <string>
#include <thread>
#include <vector>

#include "../../include/biot.h"

namespace bpk {
void set_error(const std::string& msg);
}

extern "C" {

int bp_medium_reference_borehole(int nx, int ny, int nz, float* out9) {
    if (nx < 1 || ny < 1 || nz < 1 || !out9) { bpk::set_error("bad arguments"); return BP_ERR_ARG; }
    const size_t n = (size_t)nx * ny * nz;
    float* rho = out9; float* rhof_o = out9 + n; float* M = out9 + 2 * n; float* C = out9 + 3 * n;
    float* HH = out9 + 4 * n; float* H2u = out9 + 5 * n; float* mu = out9 + 6 * n;
    float* C1 = out9 + 7 * n; float* C2 = out9 + 8 * n;
    const double porousm = 8, eta = 1.0 * pow(10.0, -3);
    for (int iz = 0; iz < nz; iz++)
        for (int iy = 0; iy < ny; iy++)
            for (int ix = 0; ix < nx; ix++) {
                const size_t i = ix + (size_t)iy * nx + (size_t)iz * nx * ny;
                if (((ix - nx / 2) * (ix - nx / 2) + (iy - ny / 2) * (iy - ny / 2)) <= 100) {
                    // fluid-filled borehole: C = M = H = H-2mu = Kf, C1 = 0, C2 = rhof
                    const float vf = 1500.0f, rf = 1000.0f;
                    const double Kf1 = rf * vf * vf;
                    rho[i] = 1000.0f; rhof_o[i] = rf; mu[i] = 0.0f;
                    C[i] = Kf1; M[i] = Kf1; HH[i] = Kf1; H2u[i] = Kf1;
                    C1[i] = 0.0f; C2[i] = rf;
                } else {
                    const float vp = 4000.0f, vs = 2700.0f, rhos = 2650.0f, rf = 1000.0f, vf = 1500.0f;
                    const double por = 0.1, perm = 2 * pow(10.0, -12), tao = 3.0;
                    const float rhov = (1 - por) * rhos + por * rf;
                    const float muv = (1 - por) * rhos * vs * vs;
                    const double Kb1 = rhos * (1 - por) * (vp * vp - vs * vs * 4.0 / 3.0);
                    const double Ks1 = rhos * (vp * vp - vs * vs * 4.0 / 3.0);
                    const double Kf1 = rf * vf * vf;
                    const double a1 = 1 - Kb1 / Ks1;
                    M[i] = Kf1 * Ks1 / (por * Ks1 + (a1 - por) * Kf1);
                    HH[i] = a1 * a1 * M[i] + Kb1 + muv * 4.0 / 3.0;
                    H2u[i] = HH[i] - 2 * muv;
                    C[i] = M[i] * a1;
                    C1[i] = eta / perm;
                    C2[i] = (1 + 2 / porousm) * tao * rf / por;
                    rho[i] = rhov; rhof_o[i] = rf; mu[i] = muv;
                }
            }
    return BP_OK;
}

// Biot coefficients from moduli, following the formation branch of
// create_model (Float/main.cu:1635-1650): alpha = 1 - Kb/Ks,
// M = Kf Ks / (phi Ks + (alpha - phi) Kf), H = alpha^2 M + Kb + 4 mu / 3,
// C = alpha M, C1 = eta / kappa, C2 = (1 + 2/m) tau rhof / phi.
int bp_biot_from_moduli(double Ks, double Kb, double mu, double Kf, double rhos, double rhof, double phi,
                        double tort, double eta, double kappa, double m_shape, double out9[9]) {
    if (!out9 || !(Ks > 0) || !(Kf > 0) || !(phi > 0) || !(phi <= 1) || !(kappa > 0) || !(m_shape > 0)) {
        bpk::set_error("bad medium parameters");
        return BP_ERR_ARG;
    }
    const double alpha = 1 - Kb / Ks;
    const double M = Kf * Ks / (phi * Ks + (alpha - phi) * Kf);
    const double H = alpha * alpha * M + Kb + mu * 4.0 / 3.0;
    out9[0] = (1 - phi) * rhos + phi * rhof;
    out9[1] = rhof;
    out9[2] = M;
    out9[3] = alpha * M;
    out9[4] = H;
    out9[5] = H - 2 * mu;
    out9[6] = mu;
    out9[7] = eta / kappa;
    out9[8] = (1 + 2 / m_shape) * tort * rhof / phi;
    return BP_OK;
}

// Fast P velocity of one cell: largest root of
// det([[H, C], [C, M]] - v^2 [[rho, rhof], [rhof, C2]]) = 0 (the frictionless,
// high-frequency limit bounds every wave speed of the discrete system); a
// fluid cell (singular mass matrix) uses sqrt(H / rho).
static double cell_vmax(double rho, double rhof, double M, double C, double H, double C2) {
    double v2 = rho > 0 ? H / rho : 0;
    const double a = rho * C2 - rhof * rhof;
    if (a > 1e-9 * std::fabs(rho * C2)) {
        const double b = -(H * C2 + M * rho - 2 * C * rhof);
        const double c = H * M - C * C;
        double disc = b * b - 4 * a * c;
        if (disc < 0) disc = 0;
        const double l = (-b + std::sqrt(disc)) / (2 * a);
        if (l > v2) v2 = l;
    }
    return std::sqrt(v2 > 0 ? v2 : 0);
}

int bp_cfl_limit(const bp_config* cfg, const bp_medium* m, double* dt_max, double* vmax_out) {
    if (!cfg || !m || !m->rho || !m->rhof || !m->M || !m->C || !m->H || !m->C2 || !dt_max) {
        bpk::set_error("bad arguments");
        return BP_ERR_ARG;
    }
    const size_t n = (size_t)cfg->nx * (cfg->dim == 3 ? cfg->ny : 1) * cfg->nz;
    // The scan runs on host threads in contiguous ranges; a cell whose six
    // inputs equal the previous cell's reuses its velocity (layered and
    // blocky media repeat along x), which changes no result.
    auto scan = [m](size_t lo, size_t hi) {
        double vmax = 0, v = 0;
        float last[6] = {NAN, NAN, NAN, NAN, NAN, NAN};
        for (size_t i = lo; i < hi; i++) {
            const float in[6] = {m->rho[i], m->rhof[i], m->M[i], m->C[i], m->H[i], m->C2[i]};
            if (!(in[0] == last[0] && in[1] == last[1] && in[2] == last[2] && in[3] == last[3] &&
                  in[4] == last[4] && in[5] == last[5])) {
                v = cell_vmax(in[0], in[1], in[2], in[3], in[4], in[5]);
                std::copy(in, in + 6, last);
            }
            if (v > vmax) vmax = v;
        }
        return vmax;
    };
    const size_t chunk = (size_t)1 << 18;
    const int nthr = (int)std::min<size_t>(std::max(1u, std::min(std::thread::hardware_concurrency(), 32u)),
                                           (n + chunk - 1) / chunk);
    double vmax = 0;
    if (nthr <= 1) {
        vmax = scan(0, n);
    } else {
        std::vector<double> part(nthr, 0.0);
        std::vector<std::thread> pool;
        const size_t per = (n + nthr - 1) / nthr;
        for (int t = 0; t < nthr; t++)
            pool.emplace_back([&, t] { part[t] = scan(std::min(n, t * per), std::min(n, (t + 1) * per)); });
        for (auto& th : pool) th.join();
        vmax = *std::max_element(part.begin(), part.end());
    }
    const double stencil = cfg->order == 4 ? (9.0 / 8.0 + 1.0 / 24.0) : 1.0;
    *dt_max = vmax > 0 ? cfg->dx / (vmax * std::sqrt((double)cfg->dim) * stencil) : 1e30;
    if (vmax_out) *vmax_out = vmax;
    return BP_OK;
}

}  // extern "C"
