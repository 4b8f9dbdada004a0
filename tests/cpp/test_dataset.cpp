// SIFT-style directory -> DatasetIrisa -> IndexBF search -> Dataset::evaluate,
// through the C++ drop-in headers.  Prints "cpp dataset ok" on success.
#include <cmath>
#include <cstdio>
#include <string>
#include <vector>

#include "curplsh/dataset.h"
#include "curplsh/device_resources.h"
#include "curplsh/index_bf.h"

int main(int argc, char** argv) {
  if (argc < 2) return 2;
  const std::string dir = argv[1];
  const int nb = 3000, nq = 40, d = 32, k = 10;
  std::vector<float> base((size_t)nb * d), query((size_t)nq * d);
  unsigned s = 12345u;
  auto rnd = [&]() { s = s * 1664525u + 1013904223u; return (float)((s >> 8) & 0xFFFF) / 65536.f; };
  for (auto& v : base) v = rnd();
  for (auto& v : query) v = rnd();
  std::vector<int> gt((size_t)nq * k);
  for (int q = 0; q < nq; ++q) {  // brute-force ground truth, lower row first on ties
    std::vector<std::pair<double, int>> dd(nb);
    for (int i = 0; i < nb; ++i) {
      double acc = 0;
      for (int j = 0; j < d; ++j) {
        const double t = (double)query[(size_t)q * d + j] - base[(size_t)i * d + j];
        acc += t * t;
      }
      dd[i] = {acc, i};
    }
    std::partial_sort(dd.begin(), dd.begin() + k, dd.end());
    for (int j = 0; j < k; ++j) gt[(size_t)q * k + j] = dd[j].second;
  }
  curplsh::helper::saveXvecsData<float, int>((dir + "/sift_base.fvecs").c_str(), base.data(), nb, d);
  curplsh::helper::saveXvecsData<float, int>((dir + "/sift_query.fvecs").c_str(), query.data(), nq, d);
  curplsh::helper::saveXvecsData<int, int>((dir + "/sift_groundtruth.ivecs").c_str(), gt.data(), nq, k);

  curplsh::DatasetSIFT ds(dir.c_str(), curplsh::MemorySpace::Device);
  if (ds.getNumBase() != nb || ds.getNumQuery() != nq || ds.getDimension() != d || ds.getGroundTruthK() != k) {
    std::printf("bad dataset shape\n");
    return 1;
  }
  curplsh::DeviceResources res;
  curplsh::IndexBFConfig cfg;
  curplsh::IndexBF index(&res, d, cfg);
  index.add(ds.getNumBase(), ds.getBase());
  int* idx = nullptr;
  float* dist = nullptr;
  cudaMalloc(&idx, sizeof(int) * nq * k);
  cudaMalloc(&dist, sizeof(float) * nq * k);
  index.search(ds.getNumQuery(), ds.getQuery(), k, idx, dist);
  std::vector<int> diff(nq);
  const float recall = ds.evaluate(idx, diff.data());
  cudaFree(idx);
  cudaFree(dist);
  std::printf("recall %.4f\n", recall);
  if (std::fabs(recall - 1.f) > 1e-6f) return 1;
  std::printf("cpp dataset ok\n");
  return 0;
}
