// Self-test of the public GPM step library (include/dumato_b200_gpm.cuh) against host
// results: for virtual warps of 8, 16 and 32 lanes, every group intersects its own pair of
// sorted lists (merge and probe regimes, empty lists included), counts the intersection,
// filters, and aggregates counters and a key histogram. Prints "gpm selftest ok" and exits 0
// when every result matches.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <random>
#include <vector>

#include "dumato_b200_gpm.cuh"

constexpr int CAP = 512;  // ints per list

template <int W>
__global__ void gpm_kernel(const int* A, const int* na, const int* B, const int* nb, int n_pairs, int* out,
                           int* n_out, int* n_count, int* filt, int* n_filt, unsigned long long* total,
                           unsigned* hist) {
  const int pair = (blockIdx.x * blockDim.x + threadIdx.x) / W;
  if (pair >= n_pairs) return;  // whole groups leave together (blockDim is a multiple of 32)
  const int* a = A + (size_t)pair * CAP;
  const int* b = B + (size_t)pair * CAP;
  const int m = dm_gpm::extend_intersect<W>(a, na[pair], b, nb[pair], out + (size_t)pair * CAP);
  const int c = dm_gpm::intersect_count<W>(a, na[pair], b, nb[pair]);
  const int f = dm_gpm::filter<W>(a, na[pair], filt + (size_t)pair * CAP, [](int x) { return x % 3 == 0; });
  if (dm_gpm::Group<W>::lane() == 0) {
    n_out[pair] = m;
    n_count[pair] = c;
    n_filt[pair] = f;
  }
  dm_gpm::aggregate_counter<W>(total, (unsigned long long)(dm_gpm::Group<W>::lane() + 1));
  for (int i0 = 0; i0 < na[pair]; i0 += W) {
    const int i = i0 + dm_gpm::Group<W>::lane();
    dm_gpm::aggregate_pattern<W>(hist, i < na[pair] ? a[i] % 16 : 0, i < na[pair]);
  }
}

#define CK(x)                                                               \
  do {                                                                      \
    cudaError_t e = (x);                                                    \
    if (e != cudaSuccess) {                                                 \
      std::printf("CUDA error %s at %s:%d\n", cudaGetErrorString(e), __FILE__, __LINE__); \
      return 1;                                                             \
    }                                                                       \
  } while (0)

template <int W>
int run(std::mt19937& rng) {
  const int n_pairs = 96;
  std::vector<int> A((size_t)n_pairs * CAP), B((size_t)n_pairs * CAP), na(n_pairs), nb(n_pairs);
  for (int p = 0; p < n_pairs; ++p) {
    const int la = p % 7 == 0 ? 0 : (int)(rng() % 200);
    const int lb = p % 5 == 0 ? (int)(rng() % CAP) : (int)(rng() % 200);  // long B: probe regime
    std::vector<int> x, y;
    const int range = 300 + (int)(rng() % 400);
    for (int i = 0; i < la; ++i) x.push_back((int)(rng() % range));
    for (int i = 0; i < lb; ++i) y.push_back((int)(rng() % range));
    std::sort(x.begin(), x.end());
    x.erase(std::unique(x.begin(), x.end()), x.end());
    std::sort(y.begin(), y.end());
    y.erase(std::unique(y.begin(), y.end()), y.end());
    na[p] = (int)x.size();
    nb[p] = (int)y.size();
    std::copy(x.begin(), x.end(), A.begin() + (size_t)p * CAP);
    std::copy(y.begin(), y.end(), B.begin() + (size_t)p * CAP);
  }
  int *dA, *dB, *dna, *dnb, *dout, *dno, *dnc, *dfilt, *dnf;
  unsigned long long* dtot;
  unsigned* dhist;
  CK(cudaMalloc(&dA, sizeof(int) * A.size()));
  CK(cudaMalloc(&dB, sizeof(int) * B.size()));
  CK(cudaMalloc(&dna, sizeof(int) * n_pairs));
  CK(cudaMalloc(&dnb, sizeof(int) * n_pairs));
  CK(cudaMalloc(&dout, sizeof(int) * A.size()));
  CK(cudaMalloc(&dfilt, sizeof(int) * A.size()));
  CK(cudaMalloc(&dno, sizeof(int) * n_pairs));
  CK(cudaMalloc(&dnc, sizeof(int) * n_pairs));
  CK(cudaMalloc(&dnf, sizeof(int) * n_pairs));
  CK(cudaMalloc(&dtot, sizeof(unsigned long long)));
  CK(cudaMalloc(&dhist, sizeof(unsigned) * 16));
  CK(cudaMemcpy(dA, A.data(), sizeof(int) * A.size(), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(dB, B.data(), sizeof(int) * B.size(), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(dna, na.data(), sizeof(int) * n_pairs, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(dnb, nb.data(), sizeof(int) * n_pairs, cudaMemcpyHostToDevice));
  CK(cudaMemset(dtot, 0, sizeof(unsigned long long)));
  CK(cudaMemset(dhist, 0, sizeof(unsigned) * 16));
  const int threads = 128;
  const int blocks = (n_pairs * W + threads - 1) / threads;
  gpm_kernel<W><<<blocks, threads>>>(dA, dna, dB, dnb, n_pairs, dout, dno, dnc, dfilt, dnf, dtot, dhist);
  CK(cudaGetLastError());
  CK(cudaDeviceSynchronize());
  std::vector<int> out(A.size()), filt(A.size()), no(n_pairs), nc(n_pairs), nf(n_pairs);
  unsigned long long tot = 0;
  std::vector<unsigned> hist(16);
  CK(cudaMemcpy(out.data(), dout, sizeof(int) * out.size(), cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(filt.data(), dfilt, sizeof(int) * filt.size(), cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(no.data(), dno, sizeof(int) * n_pairs, cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(nc.data(), dnc, sizeof(int) * n_pairs, cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(nf.data(), dnf, sizeof(int) * n_pairs, cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(&tot, dtot, sizeof(tot), cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(hist.data(), dhist, sizeof(unsigned) * 16, cudaMemcpyDeviceToHost));
  int bad = 0;
  std::vector<unsigned> want_hist(16, 0);
  for (int p = 0; p < n_pairs; ++p) {
    const int* a = A.data() + (size_t)p * CAP;
    const int* b = B.data() + (size_t)p * CAP;
    std::vector<int> want, wf;
    std::set_intersection(a, a + na[p], b, b + nb[p], std::back_inserter(want));
    for (int i = 0; i < na[p]; ++i) {
      if (a[i] % 3 == 0) wf.push_back(a[i]);
      want_hist[a[i] % 16]++;
    }
    if (no[p] != (int)want.size() || nc[p] != (int)want.size() ||
        !std::equal(want.begin(), want.end(), out.begin() + (size_t)p * CAP))
      ++bad;
    if (nf[p] != (int)wf.size() || !std::equal(wf.begin(), wf.end(), filt.begin() + (size_t)p * CAP)) ++bad;
  }
  const unsigned long long want_tot = (unsigned long long)n_pairs * W * (W + 1) / 2;
  if (tot != want_tot) ++bad;
  if (hist != want_hist) ++bad;
  cudaFree(dA);
  cudaFree(dB);
  cudaFree(dna);
  cudaFree(dnb);
  cudaFree(dout);
  cudaFree(dfilt);
  cudaFree(dno);
  cudaFree(dnc);
  cudaFree(dnf);
  cudaFree(dtot);
  cudaFree(dhist);
  std::printf("W=%d: %s\n", W, bad ? "MISMATCH" : "ok");
  return bad ? 2 : 0;
}

int main() {
  std::mt19937 rng(12345);
  int rc = run<8>(rng);
  rc = rc ? rc : run<16>(rng);
  rc = rc ? rc : run<32>(rng);
  if (rc == 0) std::printf("gpm selftest ok\n");
  return rc;
}
