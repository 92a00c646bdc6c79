// relion_dropin.cpp -- drives libb200d2 through the reference harness's C++
// API (include/b200d2_relion.hpp) the way the reference's src/main.cu does:
// projector and particle read from the reference's .dat formats, then
//   runDiff2KernelCoarse (FP32), runDiff2KernelCoarseDouble (FP64) and the
//   optimised functor on the filtered image (tensor cores),
// each accumulating onto the file's initial diff2s.  Prints one JSON line with
// the maximum relative differences to the FP64 result; exit status 1 when the
// FP32 drop-in exceeds 1e-5 or the functor exceeds 1e-5.
//
//   relion_dropin <projector.dat> <coarse_data.dat>
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <fstream>
#include <vector>

#include "b200d2_relion.hpp"

namespace {

template <typename T>
T* to_device(const std::vector<T>& h) {
  T* d = nullptr;
  if (cudaMalloc(&d, sizeof(T) * (h.empty() ? 1 : h.size())) != cudaSuccess) throw std::runtime_error("cudaMalloc");
  if (!h.empty()) cudaMemcpy(d, h.data(), sizeof(T) * h.size(), cudaMemcpyHostToDevice);
  return d;
}

template <typename T>
std::vector<T> to_host(const T* d, size_t n) {
  std::vector<T> h(n);
  cudaMemcpy(h.data(), d, sizeof(T) * n, cudaMemcpyDeviceToHost);
  return h;
}

template <typename T>
double max_rel(const std::vector<T>& a, const std::vector<double>& ref) {
  double m = 0.0;
  for (size_t i = 0; i < a.size(); ++i)
    if (std::fabs(ref[i]) > 1e-12) m = std::fmax(m, std::fabs((double)a[i] - ref[i]) / std::fabs(ref[i]));
  return m;
}

}  // namespace

int main(int argc, char** argv) {
  if (argc < 3) {
    std::fprintf(stderr, "usage: %s projector.dat coarse_data.dat\n", argv[0]);
    return 2;
  }
  try {
    AccProjector proj;
    proj.constructFromFile(argv[1]);

    // CreateCoarseParamFromFile layout (reference src/main.cu:153-191)
    std::ifstream f(argv[2], std::ios::binary);
    int hdr[7];
    f.read(reinterpret_cast<char*>(hdr), sizeof(hdr));
    const int xdim = hdr[0], ydim = hdr[1], zdim = hdr[2], rmax = hdr[3], T = hdr[4], O = hdr[5], N = hdr[6];
    std::vector<float> eulers(9 * (size_t)O), trans(2 * (size_t)T), fimg(2 * (size_t)N), corr(N),
        diff2s((size_t)O * T);
    f.read(reinterpret_cast<char*>(eulers.data()), sizeof(float) * eulers.size());
    f.read(reinterpret_cast<char*>(trans.data()), sizeof(float) * trans.size());
    f.read(reinterpret_cast<char*>(fimg.data()), sizeof(float) * fimg.size());
    f.read(reinterpret_cast<char*>(corr.data()), sizeof(float) * corr.size());
    f.read(reinterpret_cast<char*>(diff2s.data()), sizeof(float) * diff2s.size());
    if (!f) throw std::runtime_error("short coarse_data file");

    AccProjectorKernel k = AccProjectorKernel::makeKernel(proj, xdim, ydim, zdim, rmax);
    cudaStream_t stream;
    cudaStreamCreate(&stream);
    float* d_eul = to_device(eulers);
    float* d_trans = to_device(trans);
    float* d_fimg = to_device(fimg);
    float* d_corr = to_device(corr);
    float* d_out32 = to_device(diff2s);
    std::vector<double> init64(diff2s.begin(), diff2s.end());
    double* d_out64 = to_device(init64);

    runDiff2KernelCoarse(k, d_trans, d_trans + T, nullptr, d_corr, d_fimg, d_fimg + N, d_eul, d_out32, 1.f, O, T,
                         N, stream, false, false);
    // the same call with the tensor-core pipeline behind it (BF16x3)
    float* d_outbf = to_device(diff2s);
    const int prev = setCoarsePrecision(B200D2_PREC_BF16X3);
    runDiff2KernelCoarse(k, d_trans, d_trans + T, nullptr, d_corr, d_fimg, d_fimg + N, d_eul, d_outbf, 1.f, O, T,
                         N, stream, false, false);
    setCoarsePrecision(prev);
    runDiff2KernelCoarseDouble(k, d_trans, d_trans + T, nullptr, d_corr, d_fimg, d_fimg + N, d_eul, d_out64, 1.f,
                               O, T, N, stream, false, false);

    // FilterCoarseParamImage (reference src/main.cu:88-151): in-radius first
    std::vector<float> fre(N), fim(N), fco(N), cxy(2 * (size_t)N);
    int ps = 0, pe = N - 1;
    for (int i = 0; i < N; ++i) {
      int x = i % k.imgX, y = i / k.imgX;
      if (y > k.maxR) y -= k.imgY;
      float r2 = (float)(x * x + y * y) * k.padding_factor;
      r2 = r2 * k.padding_factor;
      const int d = (r2 <= (float)k.maxR2_padded) ? ps++ : pe--;
      fre[d] = fimg[i];
      fim[d] = fimg[N + i];
      fco[d] = corr[i];
      cxy[2 * d] = (float)x;
      cxy[2 * d + 1] = (float)y;
    }
    float* d_fre = to_device(fre);
    float* d_fim = to_device(fim);
    float* d_fco = to_device(fco);
    float* d_cxy = to_device(cxy);
    float* d_outtc = to_device(diff2s);
    CoarseMatrixKernelIm2colSplitImgBCFProjOverlapTransDBNfuse<> fn(T, O, ps, N, 148);
    const size_t wsb = fn.get_workspace_size_bytes();
    uint32_t* d_ws = nullptr;
    if (cudaMalloc(&d_ws, wsb) != cudaSuccess) throw std::runtime_error("workspace");
    fn.run(d_eul, d_trans, d_trans + T, d_fre, d_fim, k, d_fco, d_outtc, d_outtc, stream, d_cxy, d_ws);
    // do_CC: the cross-correlation score, against its FP64 sum
    float* d_cc = to_device(diff2s);
    std::vector<double> zero64((size_t)O * T, 0.0);
    double* d_cc64 = to_device(zero64);
    runDiff2KernelCoarse(k, d_trans, d_trans + T, nullptr, d_corr, d_fimg, d_fimg + N, d_eul, d_cc, 1.f, O, T, N,
                         stream, true, false);
    if (b200d2_diff2_coarse_cc_f64(&k.view, d_trans, d_trans + T, d_corr, d_fimg, d_fimg + N, d_eul, d_cc64, O, T,
                                   N, stream) != B200D2_OK)
      throw std::runtime_error("cc_f64");
    if (cudaStreamSynchronize(stream) != cudaSuccess) throw std::runtime_error("stream");

    const size_t n = (size_t)O * T;
    const auto o32 = to_host(d_out32, n);
    const auto o64 = to_host(d_out64, n);
    const auto otc = to_host(d_outtc, n);
    const auto obf = to_host(d_outbf, n);
    const auto occ = to_host(d_cc, n);
    const auto occ64 = to_host(d_cc64, n);
    const double e32 = max_rel(o32, o64), etc = max_rel(otc, o64), ecc = max_rel(occ, occ64),
                 ebf = max_rel(obf, o64);
    std::printf("{\"O\": %d, \"T\": %d, \"N_img\": %d, \"filtered\": %d, \"workspace_bytes\": %zu, "
                "\"fp32_vs_fp64_max_rel\": %.3e, \"functor_vs_fp64_max_rel\": %.3e, "
                "\"cc_fp32_vs_fp64_max_rel\": %.3e, \"bf16x3_dropin_vs_fp64_max_rel\": %.3e}\n",
                O, T, N, ps, wsb, e32, etc, ecc, ebf);
    for (void* p : {(void*)d_eul, (void*)d_trans, (void*)d_fimg, (void*)d_corr, (void*)d_out32, (void*)d_out64,
                    (void*)d_fre, (void*)d_fim, (void*)d_fco, (void*)d_cxy, (void*)d_outtc, (void*)d_ws,
                    (void*)d_cc, (void*)d_cc64, (void*)d_outbf})
      cudaFree(p);
    cudaStreamDestroy(stream);
    return (e32 <= 1e-5 && etc <= 1e-5 && ecc <= 1e-5 && ebf <= 1e-5) ? 0 : 1;
  } catch (const std::exception& e) {
    std::fprintf(stderr, "error: %s\n", e.what());
    return 3;
  }
}
