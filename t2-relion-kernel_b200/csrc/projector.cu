// projector.cu -- the resident reference projector (padded Hermitian-half
// Fourier volume) and its kernel-side view.
//
// Replaces AccProjector::setMdlDim / initMdl / clear / constructFromFile
// (src/acc_projector_impl.h:10-216, 300-356) and AccProjectorKernel::makeKernel
// (src/acc_projectorkernel_impl.h:410-433) of the reference harness.
//
// HBM layout: the texture representation is two single-channel float
// cudaArrays (real, imaginary) with linear filtering, clamp addressing and
// unnormalised coordinates, exactly as the reference creates them, so that the
// texture unit interpolates with the same 8-bit weights.  The linear
// representation is two dense [mdlZ][mdlY][mdlX] float arrays read by the
// software trilinear; a C2-size volume (130 x 259 x 259) is 70 MB per
// representation and stays resident in the 126 MB L2 while a batch runs.
#include <cuda_runtime.h>

#include <atomic>

#include <cstdio>
#include <cstring>
#include <vector>

#include "common.cuh"

struct b200d2_projector {
  int mdlX = 0, mdlY = 0, mdlZ = 0, mdlInitY = 0, mdlInitZ = 0, mdlMaxR = 0;
  float padding_factor = 0.f;
  cudaArray_t arr_re = nullptr, arr_im = nullptr, arr_c = nullptr;
  cudaTextureObject_t tex_re = 0, tex_im = 0, tex_c = 0;
  float* lin_re = nullptr;
  float* lin_im = nullptr;
  int device = 0;
};

namespace {

void release(b200d2_projector* p) {
  if (!p) return;
  if (p->tex_re) cudaDestroyTextureObject(p->tex_re);
  if (p->tex_im) cudaDestroyTextureObject(p->tex_im);
  if (p->tex_c) cudaDestroyTextureObject(p->tex_c);
  if (p->arr_c) cudaFreeArray(p->arr_c);
  p->tex_c = 0;
  p->arr_c = nullptr;
  if (p->arr_re) cudaFreeArray(p->arr_re);
  if (p->arr_im) cudaFreeArray(p->arr_im);
  if (p->lin_re) cudaFree(p->lin_re);
  if (p->lin_im) cudaFree(p->lin_im);
  p->tex_re = p->tex_im = 0;
  p->arr_re = p->arr_im = nullptr;
  p->lin_re = p->lin_im = nullptr;
}

int upload_array(cudaArray_t* arr, cudaTextureObject_t* tex, const float* h,
                 int X, int Y, int Z) {
  cudaChannelFormatDesc desc =
      cudaCreateChannelDesc(32, 0, 0, 0, cudaChannelFormatKindFloat);
  cudaExtent ext = make_cudaExtent(X, Y, Z);
  B200D2_CUDA_TRY(cudaMalloc3DArray(arr, &desc, ext));
  cudaMemcpy3DParms cp;
  memset(&cp, 0, sizeof(cp));
  cp.extent = ext;
  cp.kind = cudaMemcpyHostToDevice;
  cp.dstArray = *arr;
  cp.srcPtr = make_cudaPitchedPtr(const_cast<float*>(h), X * sizeof(float), X, Y);
  B200D2_CUDA_TRY(cudaMemcpy3D(&cp));
  cudaResourceDesc rd;
  memset(&rd, 0, sizeof(rd));
  rd.resType = cudaResourceTypeArray;
  rd.res.array.array = *arr;
  cudaTextureDesc td;
  memset(&td, 0, sizeof(td));
  td.filterMode = cudaFilterModeLinear;
  td.readMode = cudaReadModeElementType;
  td.normalizedCoords = 0;
  for (int i = 0; i < 3; ++i) td.addressMode[i] = cudaAddressModeClamp;
  B200D2_CUDA_TRY(cudaCreateTextureObject(tex, &rd, &td, nullptr));
  return B200D2_OK;
}

// The same volume as one float2 (re, im) array: a projection sample is one
// texture fetch instead of two.  The filtering hardware applies the same
// weights to both channels, so each channel equals the single-channel
// texture's value.
int upload_array2(cudaArray_t* arr, cudaTextureObject_t* tex, const float* h_re, const float* h_im, int X, int Y,
                  int Z) {
  const size_t n = (size_t)X * Y * Z;
  std::vector<float2> h(n);
  for (size_t i = 0; i < n; ++i) h[i] = make_float2(h_re[i], h_im[i]);
  cudaChannelFormatDesc desc = cudaCreateChannelDesc(32, 32, 0, 0, cudaChannelFormatKindFloat);
  cudaExtent ext = make_cudaExtent(X, Y, Z);
  B200D2_CUDA_TRY(cudaMalloc3DArray(arr, &desc, ext));
  cudaMemcpy3DParms cp;
  memset(&cp, 0, sizeof(cp));
  cp.extent = ext;
  cp.kind = cudaMemcpyHostToDevice;
  cp.dstArray = *arr;
  cp.srcPtr = make_cudaPitchedPtr(h.data(), X * sizeof(float2), X, Y);
  B200D2_CUDA_TRY(cudaMemcpy3D(&cp));
  cudaResourceDesc rd;
  memset(&rd, 0, sizeof(rd));
  rd.resType = cudaResourceTypeArray;
  rd.res.array.array = *arr;
  cudaTextureDesc td;
  memset(&td, 0, sizeof(td));
  td.filterMode = cudaFilterModeLinear;
  td.readMode = cudaReadModeElementType;
  td.normalizedCoords = 0;
  for (int i = 0; i < 3; ++i) td.addressMode[i] = cudaAddressModeClamp;
  B200D2_CUDA_TRY(cudaCreateTextureObject(tex, &rd, &td, nullptr));
  return B200D2_OK;
}

}  // namespace

namespace b200d2 {
static std::atomic<unsigned long long> g_projector_epoch{1};
unsigned long long projector_epoch() { return g_projector_epoch.load(); }
}  // namespace b200d2

extern "C" int b200d2_projector_create(int mdlX, int mdlY, int mdlZ,
                                       int mdlInitY, int mdlInitZ, int mdlMaxR,
                                       float padding_factor,
                                       const float* h_real,
                                       const float* h_imag, int use_texture,
                                       b200d2_projector** out) {
  if (!out || !h_real || !h_imag) return B200D2_ERR_INVALID;
  *out = nullptr;
  b200d2::g_projector_epoch.fetch_add(1);
  if (mdlZ == 1) mdlZ = 0;  // setMdlDim: zdim 1 means a 2D model
  if (mdlX <= 1 || mdlY <= 1 || mdlZ < 0) return B200D2_ERR_INVALID;
  if (mdlZ == 0) return B200D2_ERR_UNSUPPORTED;  // 2D references: out of scope
  if (use_texture < 0 || use_texture > 2) return B200D2_ERR_INVALID;
  if (!(padding_factor > 0.f) || mdlMaxR < 0) return B200D2_ERR_INVALID;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
    return B200D2_ERR_NO_DEVICE;
  b200d2_projector* p = new b200d2_projector();
  p->mdlX = mdlX;
  p->mdlY = mdlY;
  p->mdlZ = mdlZ;
  p->mdlInitY = mdlInitY;
  p->mdlInitZ = mdlInitZ;
  p->mdlMaxR = mdlMaxR;
  p->padding_factor = padding_factor;
  cudaGetDevice(&p->device);
  int st = B200D2_OK;
  if (use_texture == 1 || use_texture == 2) {
    st = upload_array(&p->arr_re, &p->tex_re, h_real, mdlX, mdlY, mdlZ);
    if (st == B200D2_OK)
      st = upload_array(&p->arr_im, &p->tex_im, h_imag, mdlX, mdlY, mdlZ);
    if (st == B200D2_OK)
      st = upload_array2(&p->arr_c, &p->tex_c, h_real, h_imag, mdlX, mdlY, mdlZ);
  }
  if (st == B200D2_OK && (use_texture == 0 || use_texture == 2)) {
    size_t n = (size_t)mdlX * mdlY * mdlZ;
    cudaError_t e = cudaMalloc(&p->lin_re, n * sizeof(float));
    if (e == cudaSuccess) e = cudaMalloc(&p->lin_im, n * sizeof(float));
    if (e == cudaSuccess)
      e = cudaMemcpy(p->lin_re, h_real, n * sizeof(float), cudaMemcpyHostToDevice);
    if (e == cudaSuccess)
      e = cudaMemcpy(p->lin_im, h_imag, n * sizeof(float), cudaMemcpyHostToDevice);
    st = b200d2::status_from_cuda(e);
  }
  if (st != B200D2_OK) {
    release(p);
    delete p;
    return st;
  }
  *out = p;
  return B200D2_OK;
}

extern "C" int b200d2_projector_load_dat(const char* path, int use_texture,
                                         b200d2_projector** out) {
  if (!path || !out) return B200D2_ERR_INVALID;
  FILE* f = fopen(path, "rb");
  if (!f) return B200D2_ERR_INVALID;
  int hdr[6];
  float pf = 0.f;
  int st = B200D2_ERR_INVALID;
  if (fread(hdr, sizeof(int), 6, f) == 6 && fread(&pf, sizeof(float), 1, f) == 1) {
    int X = hdr[0], Y = hdr[1], Z = hdr[2] == 1 ? 0 : hdr[2];
    size_t n = (size_t)X * Y * (Z == 0 ? 1 : Z);
    if (X > 0 && Y > 0 && n > 0 && n < ((size_t)1 << 34)) {
      std::vector<float> re(n), im(n);
      if (fread(re.data(), sizeof(float), n, f) == n &&
          fread(im.data(), sizeof(float), n, f) == n)
        st = b200d2_projector_create(X, Y, hdr[2], hdr[3], hdr[4], hdr[5], pf,
                                     re.data(), im.data(), use_texture, out);
    }
  }
  fclose(f);
  return st;
}

extern "C" int b200d2_projector_destroy(b200d2_projector* p) {
  if (!p) return B200D2_ERR_INVALID;
  b200d2::g_projector_epoch.fetch_add(1);
  release(p);
  delete p;
  return B200D2_OK;
}

extern "C" int b200d2_projector_dims(const b200d2_projector* p, int* dims,
                                     float* pf) {
  if (!p || !dims) return B200D2_ERR_INVALID;
  dims[0] = p->mdlX;
  dims[1] = p->mdlY;
  dims[2] = p->mdlZ;
  dims[3] = p->mdlInitY;
  dims[4] = p->mdlInitZ;
  dims[5] = p->mdlMaxR;
  if (pf) *pf = p->padding_factor;
  return B200D2_OK;
}

namespace {
__global__ void project_pixels_kernel(b200d2_view v, const float* __restrict__ eulers, int O,
                                      const int* __restrict__ px, const int* __restrict__ py, int K,
                                      float* __restrict__ out_re, float* __restrict__ out_im) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  const int o = blockIdx.y;
  if (k >= K || o >= O) return;
  const float* eo = eulers + (size_t)o * 9;
  const float e[6] = {eo[0], eo[1], eo[3], eo[4], eo[6], eo[7]};
  const float2 r = b200d2::project_pixel(v, (float)px[k], (float)py[k], e);
  out_re[(size_t)o * K + k] = r.x;
  out_im[(size_t)o * K + k] = r.y;
}
}  // namespace

extern "C" int b200d2_project_pixels(const b200d2_view* view, const float* d_eulers, int O,
                                     const int* d_px, const int* d_py, int K, float* d_out_re,
                                     float* d_out_im, void* stream) {
  if (!view || !d_eulers || !d_px || !d_py || !d_out_re || !d_out_im || O < 0 || K < 0)
    return B200D2_ERR_INVALID;
  if (view->interp == B200D2_INTERP_TEXTURE && (!view->tex_re || !view->tex_im)) return B200D2_ERR_INVALID;
  if (view->interp == B200D2_INTERP_LINEAR && (!view->lin_re || !view->lin_im)) return B200D2_ERR_INVALID;
  if (O == 0 || K == 0) return B200D2_OK;
  if (O > 65535) return B200D2_ERR_UNSUPPORTED;
  dim3 grid((K + 127) / 128, O);
  project_pixels_kernel<<<grid, 128, 0, (cudaStream_t)stream>>>(*view, d_eulers, O, d_px, d_py, K, d_out_re,
                                                                d_out_im);
  b200d2::count_launch();
  return b200d2::status_from_cuda(cudaGetLastError());
}

extern "C" int b200d2_projector_view(const b200d2_projector* p, int imgX,
                                     int imgY, int imgZ, int imgMaxR,
                                     int interp, b200d2_view* out) {
  if (!p || !out || imgX <= 0 || imgY <= 0 || imgMaxR < 0)
    return B200D2_ERR_INVALID;
  if (imgZ > 1) return B200D2_ERR_UNSUPPORTED;  // 3D data: out of scope
  if (interp == B200D2_INTERP_TEXTURE && !p->tex_re) return B200D2_ERR_INVALID;
  if (interp == B200D2_INTERP_LINEAR && !p->lin_re) return B200D2_ERR_INVALID;
  if (interp != B200D2_INTERP_TEXTURE && interp != B200D2_INTERP_LINEAR)
    return B200D2_ERR_INVALID;
  b200d2_view v;
  memset(&v, 0, sizeof(v));
  v.mdlX = p->mdlX;
  v.mdlXY = p->mdlX * p->mdlY;
  v.mdlZ = p->mdlZ;
  v.imgX = imgX;
  v.imgY = imgY;
  v.imgZ = imgZ;
  v.mdlInitY = p->mdlInitY;
  v.mdlInitZ = p->mdlInitZ;
  v.maxR = p->mdlMaxR >= imgMaxR ? imgMaxR : p->mdlMaxR;
  v.maxR2 = v.maxR * v.maxR;
  {  // int * float * float in float, truncated (acc_projectorkernel_impl.h:58)
    float r = (float)(v.maxR * v.maxR) * p->padding_factor;
    r = r * p->padding_factor;
    v.maxR2_padded = (int)r;
  }
  v.padding_factor = p->padding_factor;
  v.tex_re = (unsigned long long)p->tex_re;
  v.tex_im = (unsigned long long)p->tex_im;
  v.tex_c = (unsigned long long)p->tex_c;
  v.lin_re = p->lin_re;
  v.lin_im = p->lin_im;
  v.interp = interp;
  *out = v;
  return B200D2_OK;
}
