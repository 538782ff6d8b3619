// hp_output.cu -- the cell-centred fields of the reference's Tecplot file,
// computed on the device from the conserved state.
//
// src/main.F90:996-1131 (two-phase branch): velocities from the momenta, the
// pressure-equilibrium quadratic for p_g, p_p = p_g + 4 sigma / d, phi_g,
// the phase densities and temperatures, the phase blending near the
// volume-fraction limits, and the final densities from p and T.  Compiled
// without contraction and with the reference's operation order, so the
// values equal a plain FP64 evaluation of those lines.
#include <cuda_runtime.h>

#include "hp_device.h"

namespace hp {
namespace {

__global__ void k_tecplot_fields(const double* __restrict__ cu, long long ld, int ne, const int* __restrict__ perm,
                                 DevParams P, double* __restrict__ out) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= ne) return;
    const int t = perm[r];
    double c[10];
#pragma unroll
    for (int k = 0; k < 10; k++) c[k] = cu[(size_t)k * ld + t];
    double ug = c[1] / c[0], vg = c[2] / c[0], wg = c[3] / c[0];
    double up = c[6] / c[5], vp = c[7] / c[5], wp = c[8] / c[5];
    const double eg = c[4] / c[0] - 0.5 * (ug * ug + vg * vg + wg * wg);
    const double ep = c[9] / c[5] - 0.5 * (up * up + vp * vp + wp * wp);
    const double gg = P.gamag, gp = P.gamap, pinf = P.pinf, fs = P.fsd, emin = P.emin, emax = P.emax;
    const double bbb = (fs + pinf * gp) - (c[0] * (gg - 1.0) * eg) - (c[5] * (gp - 1.0) * ep);
    const double ccc = (c[0] * (gg - 1.0) * eg * (fs + pinf * gp));
    double pg = (-bbb + sqrt(bbb * bbb + 4.0 * ccc)) * 0.5;
    double pp = pg + fs;
    double phig = (c[0] * (gg - 1.0) * eg) / pg;
    double phip = 1.0 - phig;
    double rog = c[0] / phig, rop = c[5] / phip;
    double tg = pg / (rog * P.rrg);
    double tp = ((pp + pinf) * gp) / ((gp - 1.0) * rop * P.cpp);
    if (phig < emin) {
        phig = emin; phip = 1.0 - phig;
        ug = up; vg = vp; wg = wp; tg = tp; pg = pp;
    }
    if (phip < emin) {
        phip = emin; phig = 1.0 - phip;
        up = ug; vp = vg; wp = wg; tp = tg; pp = pg;
    }
    if (phig >= emin && phig <= emax) {
        const double psig = (phig - emin) / (emax - emin);
        const double f = -(psig * psig * (2.0 * psig - 3.0));
        ug = f * ug + (1.0 - f) * up; vg = f * vg + (1.0 - f) * vp; wg = f * wg + (1.0 - f) * wp;
        tg = f * tg + (1.0 - f) * tp; pg = f * pg + (1.0 - f) * pp;
    }
    if (phip >= emin && phip <= emax) {
        const double psig = (phip - emin) / (emax - emin);
        const double f = -(psig * psig * (2.0 * psig - 3.0));
        up = f * up + (1.0 - f) * ug; vp = f * vp + (1.0 - f) * vg; wp = f * wp + (1.0 - f) * wg;
        tp = f * tp + (1.0 - f) * tg; pp = f * pp + (1.0 - f) * pg;
    }
    rog = pg / (P.rrg * tg);
    rop = (pp + pinf) * gp / ((gp - 1.0) * P.cpp * tp);
    // the file's order: U V W PG PP TG UP VP WP PHIG TP ROG ROP
    const double v[13] = {ug, vg, wg, pg, pp, tg, up, vp, wp, phig, tp, rog, rop};
#pragma unroll
    for (int k = 0; k < 13; k++) out[(size_t)k * ne + r] = v[k];
}

}  // namespace

// Fields of ne elements, element r (reference order) at slot perm[r] of cu.
cudaError_t launch_tecplot_fields(const double* cu, long long ld, int ne, const int* perm, const DevParams& P,
                                  double* out, cudaStream_t st) {
    if (ne <= 0) return cudaSuccess;
    k_tecplot_fields<<<(unsigned)((ne + 255) / 256), 256, 0, st>>>(cu, ld, ne, perm, P, out);
    return cudaGetLastError();
}

}  // namespace hp
