// Kernel-only timing of the reference's Goldstein filter on a
// device-resident interferogram.  Test infrastructure: the reference arm of
// the benchmark runs it beside the reference executables.
//
// The reference source csrc/src/goldstein.cu is included where it lies (its
// main renamed); buffers and the batched cuFFT plan are set up as its
// goldstein_filter (goldstein.cu:410-461) does, and each repetition times
// goldstein_filter_cuda_host (goldstein.cu:328-408: patch extraction, two
// batched cuFFT C2C executions, smoothing, normalisation, weighting,
// overlap-add and the final copy of the filtered image to the host, which
// the function includes).  The plan creation is timed on its own.
//
// Usage: kbench_goldstein <ifg complex64 file> <nrow> <ncol> <n_win> <alpha> <reps>
// Prints one JSON line (ms, median over reps after one warm-up).
#define main ref_goldstein_main
#include "goldstein.cu"
#undef main

#include <algorithm>
#include <chrono>

int main(int argc, char *argv[]) {
  if (argc < 7) {
    std::cerr << "usage: kbench_goldstein <ifg> <nrow> <ncol> <n_win> <alpha> <reps>" << std::endl;
    return 2;
  }
  const int nrow = std::atoi(argv[2]), ncol = std::atoi(argv[3]), n_win = std::atoi(argv[4]);
  const float alpha = (float)std::atof(argv[5]);
  const int reps = std::max(1, std::atoi(argv[6]));
  if (nrow < n_win || ncol < n_win || n_win < 4) {
    std::cerr << "kbench_goldstein: image smaller than the window" << std::endl;
    return 2;
  }
  const int n_inc = n_win / 4;
  int n_win_i = (int)ceil((float)nrow / n_inc) - 3;
  int n_win_j = (int)ceil((float)ncol / n_inc) - 3;
  if (n_win_i <= 0) n_win_i = 1;
  if (n_win_j <= 0) n_win_j = 1;
  const int total_patches = n_win_i * n_win_j;
  const std::size_t patch_elements = std::size_t(total_patches) * n_win * n_win;
  const std::size_t img_size = (std::size_t)nrow * ncol;
  std::vector<float2> in(img_size), out(img_size);
  {
    std::ifstream f(argv[1], std::ios::binary);
    f.read(reinterpret_cast<char *>(in.data()), sizeof(float2) * img_size);
    if (!f) {
      std::cerr << "kbench_goldstein: short read" << std::endl;
      return 2;
    }
  }
  cufftComplex *d_in, *d_out, *d_patch;
  float *d_spec, *d_weight;
  CHECK_CUDA(cudaMalloc((void **)&d_in, img_size * sizeof(cufftComplex)));
  CHECK_CUDA(cudaMalloc((void **)&d_out, img_size * sizeof(cufftComplex)));
  CHECK_CUDA(cudaMalloc((void **)&d_patch, patch_elements * sizeof(cufftComplex)));
  CHECK_CUDA(cudaMalloc((void **)&d_spec, patch_elements * sizeof(float)));
  CHECK_CUDA(cudaMalloc((void **)&d_weight, img_size * sizeof(float)));
  CHECK_CUDA(cudaMemcpy(d_in, in.data(), img_size * sizeof(cufftComplex), cudaMemcpyHostToDevice));
  cufftHandle plan;
  int n[2] = {n_win, n_win}, inembed[2] = {n_win, n_win}, onembed[2] = {n_win, n_win};
  const auto p0 = std::chrono::steady_clock::now();
  CHECK_CUFFT(cufftPlanMany(&plan, 2, n, inembed, 1, n_win * n_win, onembed, 1, n_win * n_win, CUFFT_C2C,
                            total_patches));
  CHECK_CUDA(cudaDeviceSynchronize());
  const double plan_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - p0).count();
  cudaEvent_t a, b;
  CHECK_CUDA(cudaEventCreate(&a));
  CHECK_CUDA(cudaEventCreate(&b));
  std::vector<float> t;
  for (int rep = 0; rep <= reps; ++rep) {
    CHECK_CUDA(cudaMemset(d_weight, 0, img_size * sizeof(float)));
    CHECK_CUDA(cudaDeviceSynchronize());
    cudaEventRecord(a);
    goldstein_filter_cuda_host(d_in, d_out, out.data(), d_patch, d_spec, d_weight, plan, nrow, ncol, n_win, alpha);
    cudaEventRecord(b);
    CHECK_CUDA(cudaEventSynchronize(b));
    float ms;
    cudaEventElapsedTime(&ms, a, b);
    if (rep > 0) t.push_back(ms);
  }
  std::sort(t.begin(), t.end());
  std::printf("{\"goldstein_ms\": %.6f, \"plan_ms\": %.6f, \"patches\": %d, \"shape\": [%d, %d], \"reps\": %d}\n",
              t[t.size() / 2], plan_ms, total_patches, nrow, ncol, reps);
  cufftDestroy(plan);
  return 0;
}
