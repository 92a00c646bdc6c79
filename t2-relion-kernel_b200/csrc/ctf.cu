// ctf.cu -- batched multi-particle CTF folding.
//
// RELION scores a particle against CTF-modulated projections.  With the CTF
// folded into the particle side, the coarse kernel (src/diff2.cuh:369-537)
// sees
//   Fimg = X / CTF   (X where |CTF| <= 1e-8)      corr = Minvsigma2 * CTF^2
// so that corr/2 * |A - Fimg|^2 = Minvsigma2/2 * |CTF*A - X|^2 and the
// projections stay particle independent.  This kernel produces those inputs
// for a whole batch on the device from the raw particle transforms and each
// particle's CTF parameters.
//
// CTF model (the standard weak-phase form): at spatial frequency k (1/A),
// azimuth phi,
//   lambda = 12.2643247 / sqrt(V (1 + 0.978466e-6 V))       (A, V in volts)
//   dz     = (dU + dV)/2 + (dU - dV)/2 * cos(2 (phi - angle))
//   chi    = pi lambda dz k^2 - pi/2 Cs lambda^3 k^4 + phase_shift
//   CTF    = -(sqrt(1 - Q^2) sin(chi) + Q cos(chi)) * scale * exp(-B k^2 / 4)
// evaluated in FP64 and rounded once.  Pixel i of the half-plane image has
// coordinates (x, y) = pixel_index2coor(i) (src/diff2.cuh:182-188) and
// k = (x, y) / (ori_size * pixel_size).
#include <cuda_runtime.h>

#include "common.cuh"

namespace b200d2 {

__global__ void __launch_bounds__(256) ctf_fold_kernel(const float* __restrict__ re, const float* __restrict__ im,
                                                       long long stride, int N_img, int imgX, int imgY, int maxR,
                                                       double inv_box_A, const b200d2_ctf* __restrict__ ctf,
                                                       const float* __restrict__ minv, long long minv_stride,
                                                       float* __restrict__ fre, float* __restrict__ fim,
                                                       float* __restrict__ corr) {
  const int p = blockIdx.y;
  const b200d2_ctf c = ctf[p];
  const double volt = (double)c.voltage_kV * 1e3;
  const double lam = 12.2643247 / sqrt(volt * (1.0 + volt * 0.978466e-6));
  const double cs = (double)c.cs_mm * 1e7;
  const double q = (double)c.amp_contrast;
  const double sq = sqrt(1.0 - q * q);
  const double kpi = 3.14159265358979323846;
  const double ang = (double)c.defocus_angle_deg * (kpi / 180.0);
  const double shift = (double)c.phase_shift_deg * (kpi / 180.0);
  const double du = c.defocus_u_A, dv = c.defocus_v_A;
  const double scale = c.scale == 0.f ? 1.0 : (double)c.scale;
  const double bfac = c.bfactor;
  const long long at0 = (long long)p * stride;
  const float* mrow = minv + (long long)p * minv_stride;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N_img; i += gridDim.x * blockDim.x) {
    int x, y;
    pixel_coor(i, imgX, imgY, maxR, x, y);
    const double kx = x * inv_box_A, ky = y * inv_box_A;
    const double k2 = kx * kx + ky * ky;
    double dz = 0.5 * (du + dv);
    if (du != dv && k2 > 0.0) dz += 0.5 * (du - dv) * cos(2.0 * (atan2(ky, kx) - ang));
    const double chi = kpi * lam * dz * k2 - 0.5 * kpi * cs * lam * lam * lam * k2 * k2 + shift;
    double s, co;
    sincos(chi, &s, &co);
    double v = -(sq * s + q * co) * scale;
    if (bfac != 0.0) v *= exp(-0.25 * bfac * k2);
    const float xr = re[at0 + i], xi = im[at0 + i];
    const bool ok = fabs(v) > 1e-8;
    fre[at0 + i] = ok ? (float)((double)xr / v) : xr;
    fim[at0 + i] = ok ? (float)((double)xi / v) : xi;
    corr[at0 + i] = (float)((double)mrow[i] * v * v);
  }
}

}  // namespace b200d2

extern "C" int b200d2_ctf_fold(const float* d_real, const float* d_imag, long long img_stride, int P, int N_img,
                               int imgX, int imgY, int maxR, int ori_size, float pixel_A, const b200d2_ctf* d_ctf,
                               const float* d_minvsigma2, long long minvsigma2_stride, float* d_fimg_real,
                               float* d_fimg_imag, float* d_corr, void* stream) {
  using namespace b200d2;
  if (P < 0 || N_img < 0) return B200D2_ERR_INVALID;
  if (P == 0 || N_img == 0) return B200D2_OK;
  if (!d_real || !d_imag || !d_ctf || !d_minvsigma2 || !d_fimg_real || !d_fimg_imag || !d_corr)
    return B200D2_ERR_INVALID;
  if (img_stride < N_img || minvsigma2_stride < 0 || imgX <= 0 || imgY <= 0 || maxR < 0 || ori_size <= 0 ||
      !(pixel_A > 0.f) || (long long)imgX * imgY < N_img || P > 65535)
    return B200D2_ERR_INVALID;
  const dim3 grid((N_img + 255) / 256, P);
  ctf_fold_kernel<<<grid, 256, 0, (cudaStream_t)stream>>>(d_real, d_imag, img_stride, N_img, imgX, imgY, maxR,
                                                           1.0 / ((double)ori_size * pixel_A), d_ctf, d_minvsigma2,
                                                           minvsigma2_stride, d_fimg_real, d_fimg_imag, d_corr);
  count_launch();
  return status_from_cuda(cudaGetLastError());
}
