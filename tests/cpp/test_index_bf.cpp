// C++ drop-in check: the reference's own smoke pattern (test/test_search.cpp:12-36)
// through curplsh::IndexBF, host and tensor overloads.  Exit status 0 on success.
#include <cstdio>
#include <vector>

#include "curplsh/index_bf.h"

int main() {
  const int dim = 128, numBases = 1000, numQueries = 100, k = 10;
  std::vector<float> bases((size_t)numBases * dim), queries((size_t)numQueries * dim, 1.f);
  for (int i = 0; i < numBases; ++i)
    for (int d = 0; d < dim; ++d) bases[(size_t)i * dim + d] = (float)(i < 10 ? i : 10);
  curplsh::DeviceResources resources;
  curplsh::IndexBFConfig cfg;
  cfg.device = 0;
  curplsh::IndexBF index(&resources, dim, cfg);
  index.train(numBases, bases.data());
  index.add(numBases, bases.data());
  if (index.getNumData() != numBases || index.getDimension() != dim) return 10;
  std::vector<int> idx((size_t)numQueries * k);
  std::vector<float> dist((size_t)numQueries * k);
  index.search(numQueries, queries.data(), k, idx.data(), dist.data());
  const int want_idx[10] = {1, 0, 2, 3, 4, 5, 6, 7, 8, 9};
  const float want_dist[10] = {0, 128, 128, 512, 1152, 2048, 3200, 4608, 6272, 8192};
  for (int q = 0; q < numQueries; ++q)
    for (int j = 0; j < k; ++j)
      if (idx[q * k + j] != want_idx[j] || dist[q * k + j] != want_dist[j]) {
        std::printf("mismatch q=%d j=%d idx=%d dist=%f\n", q, j, idx[q * k + j], dist[q * k + j]);
        return 1;
      }
  // tensor overloads: device queries in, device results out
  curplsh::DeviceTensor<float, 2> dq(queries.data(), {numQueries, dim}, (cudaStream_t)0);
  cudaDeviceSynchronize();
  auto res = index.search(dq, k);
  std::vector<int> idx2((size_t)numQueries * k);
  res.second.toHost(idx2.data());
  for (size_t t = 0; t < idx2.size(); ++t)
    if (idx2[t] != idx[t]) return 2;
  // errors surface as exceptions, not aborts
  bool threw = false;
  try {
    index.search(1, queries.data(), 2000, idx.data(), dist.data());
  } catch (const curplsh::Error& e) {
    threw = e.code() == CURPLSH_ERR_INVALID_ARG;
  }
  if (!threw) return 3;
  index.reset();
  if (index.getNumData() != 0) return 4;
  std::printf("cpp drop-in ok\n");
  return 0;
}
