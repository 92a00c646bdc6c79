/*
 * diff2_oracle.c -- CPU restatement of RELION's coarse-pass diff2.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker that the CUDA path is
 * compared against (tests/, __graft_entry__.smoke(), and the CPU-baseline leg
 * of bench.py).  It is never part of the product: the library under
 * t2-relion-kernel_b200/ does not link, load or call it, and has no CPU
 * fallback.
 *
 * What it restates (file:line in the reference project Edgarrrrrr/T2-RELION-kernel):
 *   - AccProjectorKernel constructor / makeKernel: maxR = min(mdlMaxR, imgMaxR),
 *     maxR2 = maxR^2, maxR2_padded = int(maxR^2 * pf * pf)
 *       src/acc_projectorkernel_impl.h:63-75, 410-433
 *   - project3Dmodel(x, y, e0,e1,e3,e4,e6,e7): rotate a 2D Fourier pixel into
 *     the padded 3D volume, int-truncated radius test, Hermitian conjugate when
 *     xp < 0, trilinear fetch at (xp, yp - mdlInitY, zp - mdlInitZ)
 *       src/acc_projectorkernel_impl.h:178-252
 *   - no_tex3D (software trilinear, order of the lerps)
 *       src/cuda_device_utils.cuh:73-108
 *   - translatePixel: (c*re - s*im, c*im + s*re) with sincos(x*tx + y*ty)
 *       src/cuda_device_utils.cuh:110-129
 *   - pixel_index2coor: x = i % imgX, y = i / imgX, y -= imgY if y > maxR
 *       src/diff2.cuh:182-188
 *   - cuda_kernel_diff2_coarse: diff2s[o*T + t] += sum_i |ref - shift(img)|^2 * corr/2
 *     over all image_size pixels, accumulating onto the caller's buffer
 *       src/diff2.cuh:369-537
 *   - FilterCoarseParamImage: in-radius pixels first, then the rest (the
 *     outside block is filled from the end backwards)
 *       src/main.cu:88-151
 *
 * Interpolation modes.  The reference fetches the projector through a CUDA
 * texture object with cudaFilterModeLinear (src/acc_projector_impl.h:98-103).
 * The CUDA programming guide documents that linear filtering keeps each
 * weight in 9-bit fixed point with 8 fractional bits.  ORC_INTERP_TEX_*
 * therefore quantise the fractional coordinate to 1/256 before the weights are
 * formed (round-to-nearest or truncation of the fixed-point coordinate), clamp
 * the indices to the array (cudaAddressModeClamp) and form the weighted sum in
 * double.  ORC_INTERP_EXACT is the reference's no_tex3D arithmetic in double.
 *
 * FP32 coordinate arithmetic.  Coordinates are formed in float exactly as the
 * CUDA kernels of this repository form them (explicit fused multiply-adds in a
 * fixed order), so that the oracle and the GPU see identical sample positions.
 * This file must be compiled with -ffp-contract=off so that gcc does not add
 * contractions of its own.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define ORC_INTERP_EXACT 0
#define ORC_INTERP_TEX_ROUND 1
#define ORC_INTERP_TEX_TRUNC 2

typedef struct orc_projector {
  /* padded Hermitian-half Fourier volume, x fastest: [mdlZ][mdlY][mdlX] */
  int mdlX, mdlY, mdlZ, mdlInitY, mdlInitZ, mdlMaxR;
  float padding_factor;
  /* kernel view (makeKernel) */
  int imgX, imgY, imgZ, maxR, maxR2, maxR2_padded;
  const float *re;
  const float *im;
} orc_projector;

int orc_abi_version(void) { return 3; }

/* makeKernel: src/acc_projectorkernel_impl.h:410-433, constructor :63-75 */
void orc_projector_init(orc_projector *p, int mdlX, int mdlY, int mdlZ,
                        int mdlInitY, int mdlInitZ, int mdlMaxR,
                        float padding_factor, const float *re, const float *im,
                        int imgX, int imgY, int imgZ, int imgMaxR) {
  p->mdlX = mdlX;
  p->mdlY = mdlY;
  p->mdlZ = (mdlZ == 1) ? 0 : mdlZ; /* setMdlDim: zdim 1 means 2D */
  p->mdlInitY = mdlInitY;
  p->mdlInitZ = mdlInitZ;
  p->mdlMaxR = mdlMaxR;
  p->padding_factor = padding_factor;
  p->imgX = imgX;
  p->imgY = imgY;
  p->imgZ = imgZ;
  p->maxR = mdlMaxR >= imgMaxR ? imgMaxR : mdlMaxR;
  p->maxR2 = p->maxR * p->maxR;
  {
    /* int * float * float evaluated in float, then truncated to int */
    float v = (float)(p->maxR * p->maxR) * padding_factor;
    v = v * padding_factor;
    p->maxR2_padded = (int)v;
  }
  p->re = re;
  p->im = im;
}

int orc_projector_maxR(const orc_projector *p) { return p->maxR; }
int orc_projector_maxR2_padded(const orc_projector *p) { return p->maxR2_padded; }

/* pixel_index2coor: src/diff2.cuh:182-188 */
static inline void orc_pixel_coor(const orc_projector *p, long idx, int *x,
                                  int *y) {
  *x = (int)(idx % p->imgX);
  *y = (int)(idx / p->imgX);
  if (*y > p->maxR) *y -= p->imgY;
}

/* Rotated, padded coordinates in float with the fused multiply-add order used
 * by the CUDA kernels:  xp = fma(e0, x, e1*y) * pf ;
 * r2 = (int) fma(zp, zp, fma(xp, xp, yp*yp)). */
static inline void orc_rotate_f32(const orc_projector *p, int x, int y,
                                  const float *e, float *xp, float *yp,
                                  float *zp, int *r2) {
  const float fx = (float)x, fy = (float)y, pf = p->padding_factor;
  float a = fmaf(e[0], fx, e[1] * fy) * pf;
  float b = fmaf(e[3], fx, e[4] * fy) * pf;
  float c = fmaf(e[6], fx, e[7] * fy) * pf;
  float s = fmaf(c, c, fmaf(a, a, b * b));
  *xp = a;
  *yp = b;
  *zp = c;
  *r2 = (int)s;
}

static inline long orc_clampi(long v, long lo, long hi) {
  return v < lo ? lo : (v > hi ? hi : v);
}

static inline double orc_voxel(const float *mdl, const orc_projector *p, long x,
                               long y, long z) {
  x = orc_clampi(x, 0, p->mdlX - 1);
  y = orc_clampi(y, 0, p->mdlY - 1);
  z = orc_clampi(z, 0, p->mdlZ - 1);
  return (double)mdl[(z * p->mdlY + y) * p->mdlX + x];
}

/* Split a texel-space coordinate u (texture convention: sample centres at
 * integer + 0.5, so the reference passes xp + 0.5) into base index and
 * interpolation weight, with the weight quantised as the texture unit does. */
static inline void orc_tex_split(double u, int mode, long *i0, double *a) {
  double xb = u - 0.5;
  if (mode == ORC_INTERP_TEX_ROUND) {
    double q = floor(xb * 256.0 + 0.5);
    double fl = floor(q / 256.0);
    *i0 = (long)fl;
    *a = (q - fl * 256.0) / 256.0;
  } else if (mode == ORC_INTERP_TEX_TRUNC) {
    double q = floor(xb * 256.0);
    double fl = floor(q / 256.0);
    *i0 = (long)fl;
    *a = (q - fl * 256.0) / 256.0;
  } else {
    double fl = floor(xb);
    *i0 = (long)fl;
    *a = xb - fl;
  }
}

/* Measured on the B200 (tests/test_gpu_texture.py): the 1D behaviour above
 * (fraction rounded half-up to 1/256, weight 1.0 reachable) is exact, and
 * the eight 3D corner weights are multiples of 1/256 summing to exactly one,
 * but the hardware rounds them jointly in a way this separable model does
 * not reproduce; per sample the difference is up to ~1e-2 of the voxel scale,
 * on diff2 up to ~2e-4 relative.  Parity of the texture path is therefore
 * pinned against the reference's own kernels and against the texture unit's
 * own samples (orc_diff2_from_projections), not against this model. */

/* Trilinear fetch of one component at texel coordinates (u, v, w), where
 * u = xp + 0.5, v = yp - mdlInitY + 0.5, w = zp - mdlInitZ + 0.5 exactly as
 * the reference forms them in float before tex3D
 * (src/acc_projectorkernel_impl.h:232-250). */
static double orc_trilinear(const float *mdl, const orc_projector *p, float u,
                            float v, float w, int mode) {
  long x0, y0, z0;
  double fx, fy, fz;
  orc_tex_split((double)u, mode, &x0, &fx);
  orc_tex_split((double)v, mode, &y0, &fy);
  orc_tex_split((double)w, mode, &z0, &fz);
  double d000 = orc_voxel(mdl, p, x0, y0, z0);
  double d001 = orc_voxel(mdl, p, x0 + 1, y0, z0);
  double d010 = orc_voxel(mdl, p, x0, y0 + 1, z0);
  double d011 = orc_voxel(mdl, p, x0 + 1, y0 + 1, z0);
  double d100 = orc_voxel(mdl, p, x0, y0, z0 + 1);
  double d101 = orc_voxel(mdl, p, x0 + 1, y0, z0 + 1);
  double d110 = orc_voxel(mdl, p, x0, y0 + 1, z0 + 1);
  double d111 = orc_voxel(mdl, p, x0 + 1, y0 + 1, z0 + 1);
  /* lerp order of no_tex3D: x, then y, then z */
  double dx00 = d000 + (d001 - d000) * fx;
  double dx01 = d100 + (d101 - d100) * fx;
  double dx10 = d010 + (d011 - d010) * fx;
  double dx11 = d110 + (d111 - d110) * fx;
  double dxy0 = dx00 + (dx10 - dx00) * fy;
  double dxy1 = dx01 + (dx11 - dx01) * fy;
  return dxy0 + (dxy1 - dxy0) * fz;
}

/* project3Dmodel for a 2D image into a 3D reference
 * (src/acc_projectorkernel_impl.h:178-252).  Returns 1 if inside. */
static int orc_project_one(const orc_projector *p, int x, int y, const float *e,
                           int mode, double *re, double *im) {
  float xp, yp, zp;
  int r2;
  orc_rotate_f32(p, x, y, e, &xp, &yp, &zp, &r2);
  if (r2 <= p->maxR2_padded) {
    double sign = 1.0;
    if (xp < 0) {
      xp = -xp;
      yp = -yp;
      zp = -zp;
      sign = -1.0;
    }
    yp -= (float)p->mdlInitY;
    zp -= (float)p->mdlInitZ;
    float u = xp + 0.5f, v = yp + 0.5f, w = zp + 0.5f;
    *re = orc_trilinear(p->re, p, u, v, w, mode);
    *im = sign * orc_trilinear(p->im, p, u, v, w, mode);
    return 1;
  }
  *re = 0.0;
  *im = 0.0;
  return 0;
}

/* Projection matrix for a pixel list: out[o*K + k] (row = orientation). */
void orc_project_pixels(const orc_projector *p, const float *eulers, long O,
                        const int *px, const int *py, long K, int mode,
                        double *out_re, double *out_im, int nthreads) {
  long o;
#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(static)
#endif
  for (o = 0; o < O; o++) {
    const float *e = eulers + 9 * o;
    for (long k = 0; k < K; k++)
      orc_project_one(p, px[k], py[k], e, mode, &out_re[o * K + k],
                      &out_im[o * K + k]);
  }
}

/* FP64 oracle of cuda_kernel_diff2_coarse (src/diff2.cuh:369-537):
 * diff2[o*T + t] += sum_{i < N_img} |ref_o(i) - shift_t(img)(i)|^2 * corr(i)/2
 * Projections come from orc_project_one (float coordinates, double values);
 * the phase, rotation, differences and sum are double. */
void orc_diff2_coarse_f64(const orc_projector *p, const float *eulers, long O,
                          const float *trans_x, const float *trans_y, long T,
                          const float *fre, const float *fim, const float *corr,
                          long N_img, int mode, double *diff2, int nthreads) {
  int *px = (int *)malloc(sizeof(int) * (size_t)N_img);
  int *py = (int *)malloc(sizeof(int) * (size_t)N_img);
  double *sre = (double *)malloc(sizeof(double) * (size_t)(N_img * T));
  double *sim = (double *)malloc(sizeof(double) * (size_t)(N_img * T));
  for (long i = 0; i < N_img; i++) orc_pixel_coor(p, i, &px[i], &py[i]);
  /* translatePixel in double (src/cuda_device_utils.cuh:132-151) */
  for (long t = 0; t < T; t++)
    for (long i = 0; i < N_img; i++) {
      double ph = px[i] * (double)trans_x[t] + py[i] * (double)trans_y[t];
      double s = sin(ph), c = cos(ph);
      double r = fre[i], m = fim[i];
      sre[t * N_img + i] = c * r - s * m;
      sim[t * N_img + i] = c * m + s * r;
    }
  long o;
#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 4)
#endif
  for (o = 0; o < O; o++) {
    double *ar = (double *)malloc(sizeof(double) * (size_t)N_img);
    double *ai = (double *)malloc(sizeof(double) * (size_t)N_img);
    for (long i = 0; i < N_img; i++)
      orc_project_one(p, px[i], py[i], eulers + 9 * o, mode, &ar[i], &ai[i]);
    for (long t = 0; t < T; t++) {
      const double *r = sre + t * N_img, *m = sim + t * N_img;
      double acc = 0.0;
      for (long i = 0; i < N_img; i++) {
        double dr = ar[i] - r[i], di = ai[i] - m[i];
        acc += (dr * dr + di * di) * ((double)corr[i] / 2.0);
      }
      diff2[o * T + t] += acc;
    }
    free(ar);
    free(ai);
  }
  free(px);
  free(py);
  free(sre);
  free(sim);
}

/* Same FP64 sum as orc_diff2_coarse_f64, but with the projections given
 * (prj_re/prj_im[o*N_img + i] for every image pixel i): isolates the
 * arithmetic of cuda_kernel_diff2_coarse from the interpolation. */
void orc_diff2_from_projections(const orc_projector *p, const float *prj_re,
                                const float *prj_im, long O,
                                const float *trans_x, const float *trans_y,
                                long T, const float *fre, const float *fim,
                                const float *corr, long N_img, double *diff2,
                                int nthreads) {
  long o;
#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 4)
#endif
  for (o = 0; o < O; o++) {
    for (long t = 0; t < T; t++) {
      double acc = 0.0;
      for (long i = 0; i < N_img; i++) {
        int x, y;
        orc_pixel_coor(p, i, &x, &y);
        double ph = x * (double)trans_x[t] + y * (double)trans_y[t];
        double s = sin(ph), c = cos(ph);
        double r = fre[i], m = fim[i];
        double sr = c * r - s * m, si = c * m + s * r;
        double dr = (double)prj_re[o * N_img + i] - sr;
        double di = (double)prj_im[o * N_img + i] - si;
        acc += (dr * dr + di * di) * ((double)corr[i] / 2.0);
      }
      diff2[o * T + t] += acc;
    }
  }
}

/* ---------------------------------------------------------------------------
 * FP32 port of cuda_kernel_diff2_coarse (the timed CPU baseline).
 * Same loop structure as the reference kernel: blocks of 16 orientations are
 * projected into a buffer, then for every translation each pixel is shifted
 * once (sincosf) and its difference to the 16 projections accumulated in
 * float.  Texture-weight interpolation is emulated in float.
 * ------------------------------------------------------------------------- */
static inline float orc_voxf(const float *mdl, const orc_projector *p, long x,
                             long y, long z) {
  x = orc_clampi(x, 0, p->mdlX - 1);
  y = orc_clampi(y, 0, p->mdlY - 1);
  z = orc_clampi(z, 0, p->mdlZ - 1);
  return mdl[(z * p->mdlY + y) * p->mdlX + x];
}

static inline void orc_split_f(float u, long *i0, float *a) {
  float q = floorf((u - 0.5f) * 256.0f + 0.5f);
  float fl = floorf(q * (1.0f / 256.0f));
  *i0 = (long)fl;
  *a = (q - fl * 256.0f) * (1.0f / 256.0f);
}

static float orc_trilinear_f(const float *mdl, const orc_projector *p, float u,
                             float v, float w) {
  long x0, y0, z0;
  float fx, fy, fz;
  orc_split_f(u, &x0, &fx);
  orc_split_f(v, &y0, &fy);
  orc_split_f(w, &z0, &fz);
  float d000 = orc_voxf(mdl, p, x0, y0, z0), d001 = orc_voxf(mdl, p, x0 + 1, y0, z0);
  float d010 = orc_voxf(mdl, p, x0, y0 + 1, z0), d011 = orc_voxf(mdl, p, x0 + 1, y0 + 1, z0);
  float d100 = orc_voxf(mdl, p, x0, y0, z0 + 1), d101 = orc_voxf(mdl, p, x0 + 1, y0, z0 + 1);
  float d110 = orc_voxf(mdl, p, x0, y0 + 1, z0 + 1), d111 = orc_voxf(mdl, p, x0 + 1, y0 + 1, z0 + 1);
  float dx00 = d000 + (d001 - d000) * fx, dx01 = d100 + (d101 - d100) * fx;
  float dx10 = d010 + (d011 - d010) * fx, dx11 = d110 + (d111 - d110) * fx;
  float dxy0 = dx00 + (dx10 - dx00) * fy, dxy1 = dx01 + (dx11 - dx01) * fy;
  return dxy0 + (dxy1 - dxy0) * fz;
}

static void orc_project_one_f(const orc_projector *p, int x, int y,
                              const float *e, float *re, float *im) {
  float xp, yp, zp;
  int r2;
  orc_rotate_f32(p, x, y, e, &xp, &yp, &zp, &r2);
  if (r2 <= p->maxR2_padded) {
    float sign = 1.0f;
    if (xp < 0) {
      xp = -xp;
      yp = -yp;
      zp = -zp;
      sign = -1.0f;
    }
    yp -= (float)p->mdlInitY;
    zp -= (float)p->mdlInitZ;
    *re = orc_trilinear_f(p->re, p, xp + 0.5f, yp + 0.5f, zp + 0.5f);
    *im = sign * orc_trilinear_f(p->im, p, xp + 0.5f, yp + 0.5f, zp + 0.5f);
  } else {
    *re = 0.0f;
    *im = 0.0f;
  }
}

#define ORC_EPB 16 /* D2C_EULERS_PER_BLOCK_REF3D, src/common.h:44 */

void orc_diff2_coarse_f32(const orc_projector *p, const float *eulers, long O,
                          const float *trans_x, const float *trans_y, long T,
                          const float *fre, const float *fim, const float *corr,
                          long N_img, float *diff2, int nthreads) {
  int *px = (int *)malloc(sizeof(int) * (size_t)N_img);
  int *py = (int *)malloc(sizeof(int) * (size_t)N_img);
  float *wc = (float *)malloc(sizeof(float) * (size_t)N_img);
  for (long i = 0; i < N_img; i++) {
    orc_pixel_coor(p, i, &px[i], &py[i]);
    wc[i] = corr[i] / 2;
  }
  long nblk = (O + ORC_EPB - 1) / ORC_EPB;
  long b;
#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 1)
#endif
  for (b = 0; b < nblk; b++) {
    long o0 = b * ORC_EPB;
    int ne = (int)((O - o0) < ORC_EPB ? (O - o0) : ORC_EPB);
    float *rr = (float *)malloc(sizeof(float) * (size_t)N_img * ORC_EPB);
    float *ri = (float *)malloc(sizeof(float) * (size_t)N_img * ORC_EPB);
    for (long i = 0; i < N_img; i++)
      for (int j = 0; j < ORC_EPB; j++) {
        if (j < ne)
          orc_project_one_f(p, px[i], py[i], eulers + 9 * (o0 + j),
                            &rr[i * ORC_EPB + j], &ri[i * ORC_EPB + j]);
        else
          rr[i * ORC_EPB + j] = ri[i * ORC_EPB + j] = 0.0f;
      }
    for (long t = 0; t < T; t++) {
      float acc[ORC_EPB];
      for (int j = 0; j < ORC_EPB; j++) acc[j] = 0.0f;
      const float tx = trans_x[t], ty = trans_y[t];
      for (long i = 0; i < N_img; i++) {
        float s = sinf(px[i] * tx + py[i] * ty);
        float c = cosf(px[i] * tx + py[i] * ty);
        float sr = c * fre[i] - s * fim[i];
        float si = c * fim[i] + s * fre[i];
        const float w = wc[i];
        const float *ar = rr + i * ORC_EPB, *ai = ri + i * ORC_EPB;
        for (int j = 0; j < ORC_EPB; j++) {
          float dr = ar[j] - sr, di = ai[j] - si;
          acc[j] += (dr * dr + di * di) * w;
        }
      }
      for (int j = 0; j < ne; j++) diff2[(o0 + j) * T + t] += acc[j];
    }
    free(rr);
    free(ri);
  }
  free(px);
  free(py);
  free(wc);
}

/* FilterCoarseParamImage (src/main.cu:88-151): pixels with
 * (x^2 + y^2) * pf * pf <= maxR2_padded (float test) are written from the
 * front, the others from the back.  Returns the in-radius count. */
long orc_filter_image(const orc_projector *p, const float *fre,
                      const float *fim, const float *corr, long N_img,
                      float *out_re, float *out_im, float *out_corr,
                      float *out_coor_xy) {
  long ps = 0, pe = N_img - 1;
  for (long i = 0; i < N_img; i++) {
    int x, y;
    orc_pixel_coor(p, i, &x, &y);
    float r2 = (float)(x * x + y * y) * p->padding_factor;
    r2 = r2 * p->padding_factor;
    long d;
    if (r2 <= (float)p->maxR2_padded)
      d = ps++;
    else
      d = pe--;
    out_re[d] = fre[i];
    out_im[d] = fim[i];
    out_corr[d] = corr[i];
    out_coor_xy[2 * d] = (float)x;
    out_coor_xy[2 * d + 1] = (float)y;
  }
  return ps;
}

/* Sample a [Z][Y][X] volume at texel coordinates (u, v, w) with the same
 * interpolation routine the projections use (texture-unit emulation check). */
void orc_tex_sample(const float *vol, int X, int Y, int Z, const float *uvw,
                    long n, int mode, double *out) {
  orc_projector p;
  memset(&p, 0, sizeof(p));
  p.mdlX = X;
  p.mdlY = Y;
  p.mdlZ = Z;
  for (long i = 0; i < n; i++)
    out[i] = orc_trilinear(vol, &p, uvw[3 * i], uvw[3 * i + 1], uvw[3 * i + 2],
                           mode);
}
