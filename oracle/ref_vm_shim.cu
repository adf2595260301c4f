// TEST ORACLE shim: launches the reference's own `kernel_dynamic` (src/kernel.cu,
// compiled from the reference tree with -DKER and the stand-in header ref_stub/) on
// reference-format instruction streams.  Used by the GPU parity tests only, always with
// ONE worker: a single stream carries no signal_wait, so the reference's unbounded spin
// (src/kernel.cu:1503-1509) is never entered.
#include <kernel.cu>

#include <cstdint>
#include <vector>

extern "C" int ref_vm_run(int workers, const int* words, const int* lengths, void* const* ptrs, int n_ptrs,
                          int n_signals, double* rnd_dev, long long tmp_elems, int threads) {
  if (workers != 1) return (int)cudaErrorInvalidValue;  // see header comment
  cudaError_t e = cudaSuccess;
  std::vector<int*> d_streams(workers, nullptr);
  std::vector<double*> d_tmps(workers, nullptr);
  std::vector<unsigned long long*> d_clk(workers, nullptr);
  int** d_insts = nullptr;
  void** d_ptrs = nullptr;
  int* d_comm = nullptr;
  double** d_tmp_tab = nullptr;
  unsigned long long** d_clk_tab = nullptr;
  long long at = 0;
  for (int w = 0; w < workers && e == cudaSuccess; ++w) {
    // the kernel fetches _MAX_INST_LENGTH words per instruction: pad every stream
    const size_t len = (size_t)lengths[w] + _MAX_INST_LENGTH;
    std::vector<int> padded(len, 0);
    for (int i = 0; i < lengths[w]; ++i) padded[i] = words[at + i];
    at += lengths[w];
    e = cudaMalloc(&d_streams[w], len * sizeof(int));
    if (e == cudaSuccess) e = cudaMemcpy(d_streams[w], padded.data(), len * sizeof(int), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMalloc(&d_tmps[w], sizeof(double) * (tmp_elems > 0 ? tmp_elems : 1));
    if (e == cudaSuccess) e = cudaMalloc(&d_clk[w], sizeof(unsigned long long) * len);
  }
  if (e == cudaSuccess) e = cudaMalloc(&d_insts, sizeof(int*) * workers);
  if (e == cudaSuccess) e = cudaMemcpy(d_insts, d_streams.data(), sizeof(int*) * workers, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMalloc(&d_ptrs, sizeof(void*) * n_ptrs);
  if (e == cudaSuccess) e = cudaMemcpy(d_ptrs, ptrs, sizeof(void*) * n_ptrs, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMalloc(&d_comm, sizeof(int) * (n_signals > 0 ? n_signals : 1));
  if (e == cudaSuccess) e = cudaMemset(d_comm, 0, sizeof(int) * (n_signals > 0 ? n_signals : 1));
  if (e == cudaSuccess) e = cudaMalloc(&d_tmp_tab, sizeof(double*) * workers);
  if (e == cudaSuccess) e = cudaMemcpy(d_tmp_tab, d_tmps.data(), sizeof(double*) * workers, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMalloc(&d_clk_tab, sizeof(unsigned long long*) * workers);
  if (e == cudaSuccess) e = cudaMemcpy(d_clk_tab, d_clk.data(), sizeof(void*) * workers, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) {
    kernel_dynamic<<<workers, threads>>>((const int**)d_insts, d_ptrs, d_comm, d_tmp_tab, rnd_dev, d_clk_tab);
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
  }
  for (int w = 0; w < workers; ++w) { cudaFree(d_streams[w]); cudaFree(d_tmps[w]); cudaFree(d_clk[w]); }
  cudaFree(d_insts); cudaFree(d_ptrs); cudaFree(d_comm); cudaFree(d_tmp_tab); cudaFree(d_clk_tab);
  return (int)e;
}
