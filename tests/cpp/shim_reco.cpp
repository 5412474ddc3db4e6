// The reference's reco iteration (src/tests/reco.cu:230-303) written against
// the C++ template API of include/raptr_b200.hpp: systemMatrixCalculation,
// CSRmv<float>, divides, dividesMultiplies, sum, scales.  Small geometry,
// every 301st channel, 5 iterations; writes the image to argv[1].  With
// argv[2] = "keep" the rows keep exact zeros (the reference's structure).
#include <cstdio>
#include <string>
#include <vector>

#include "raptr_b200.hpp"

typedef float val_t;
typedef DefaultVoxelGrid<val_t> VG;
typedef DefaultMeasurementSetup<val_t> MS;

#define CK(x) raptr::check_cuda((x), #x)

int main(int argc, char** argv) {
  if (argc < 2 || argc > 3) return 2;
  try {
    VG grid(-0.04f, -0.04f, -0.04f, 0.002f, 0.002f, 0.002f, 40, 40, 40);
    MS setup(-0.24f, 0.24f, 5, 13, 13, 13, 13, 36.f, 0.020f, 0.004f, 0.004f);
    const int nrays = 100;
    raptr::set_device_constants(grid, setup, nrays, 1251);
    if (argc == 3 && std::string(argv[2]) == "keep") raptr::set_sm_flags(RAPTR_SM_KEEP_ZEROS);
    const int M = 5 * 13 * 13 * 13 * 13, N = 40 * 40 * 40;
    std::vector<int> yRowId;
    for (int c = 0; c < M; c += 301) yRowId.push_back(c);
    uint32_t m = uint32_t(yRowId.size());

    int *yRowId_devi, *aEcsr, *aVxl, *aCnl, *aCsr;
    float *aVal;
    unsigned long long* nnz_devi;
    CK(cudaMalloc(&yRowId_devi, m * sizeof(int)));
    CK(cudaMemcpy(yRowId_devi, yRowId.data(), m * sizeof(int), cudaMemcpyHostToDevice));
    CK(cudaMalloc(&aEcsr, (m + 1) * sizeof(int)));
    CK(cudaMalloc(&aVxl, size_t(m) * N * sizeof(int)));  // the reference's dense bound
    CK(cudaMalloc(&aVal, size_t(m) * N * sizeof(float)));
    CK(cudaMalloc(&aCnl, sizeof(int)));
    CK(cudaMalloc(&aCsr, sizeof(int)));
    CK(cudaMalloc(&nnz_devi, sizeof(unsigned long long)));
    CK(cudaMemset(nnz_devi, 0, sizeof(unsigned long long)));
    int handle = 0, descr = 0;
    systemMatrixCalculation<val_t, uint32_t, int, unsigned long long, int>(aEcsr, aVxl, aVal, nnz_devi, aCnl, aCsr,
                                                                           yRowId_devi, &m, handle);
    unsigned long long nnz = 0;
    CK(cudaMemcpy(&nnz, nnz_devi, sizeof(nnz), cudaMemcpyDeviceToHost));

    // phantom: background 0.1, sphere r 15 mm 1.0, sphere r 8 mm at +20 mm 4.0
    std::vector<float> xt(N);
    for (int ix = 0; ix < 40; ix++)
      for (int iy = 0; iy < 40; iy++)
        for (int iz = 0; iz < 40; iz++) {
          double cx = -0.04 + (ix + 0.5) * 0.002, cy = -0.04 + (iy + 0.5) * 0.002, cz = -0.04 + (iz + 0.5) * 0.002;
          float v = 0.1f;
          if (cx * cx + cy * cy + cz * cz < 0.015 * 0.015) v = 1.0f;
          if ((cx - 0.02) * (cx - 0.02) + cy * cy + cz * cz < 0.008 * 0.008) v = 4.0f;
          xt[size_t(ix) * 1600 + iy * 40 + iz] = v;
        }
    float *x, *xx, *xtd, *y, *yt, *e, *c, *s, *ones;
    CK(cudaMalloc(&x, N * sizeof(float)));
    CK(cudaMalloc(&xx, N * sizeof(float)));
    CK(cudaMalloc(&xtd, N * sizeof(float)));
    CK(cudaMalloc(&c, N * sizeof(float)));
    CK(cudaMalloc(&s, N * sizeof(float)));
    CK(cudaMalloc(&y, m * sizeof(float)));
    CK(cudaMalloc(&yt, m * sizeof(float)));
    CK(cudaMalloc(&e, m * sizeof(float)));
    CK(cudaMalloc(&ones, m * sizeof(float)));
    CK(cudaMemcpy(xtd, xt.data(), N * sizeof(float), cudaMemcpyHostToDevice));
    std::vector<float> h1(m, 1.f), hx(N, 1.f / N);
    CK(cudaMemcpy(ones, h1.data(), m * sizeof(float), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(x, hx.data(), N * sizeof(float), cudaMemcpyHostToDevice));
    float scale = 1e4f, one = 1.f, zero = 0.f;
    CSRmv<float>()(handle, 0, int(m), N, int(nnz), &scale, descr, aVal, aEcsr, aVxl, xtd, &zero, y);  // y = 1e4 A x_true
    CSRmv<float>()(handle, 1, int(m), N, int(nnz), &one, descr, aVal, aEcsr, aVxl, ones, &zero, s);   // s = A^T 1
    float norm = sum<val_t>(s, N);
    scales<val_t>(s, val_t(1. / norm), N);
    for (int it = 0; it < 5; it++) {
      CSRmv<float>()(handle, 0, int(m), N, int(nnz), &one, descr, aVal, aEcsr, aVxl, x, &zero, yt);
      divides<val_t>(e, y, yt, int(m));
      CK(cudaMemset(c, 0, N * sizeof(float)));
      CSRmv<float>()(handle, 1, int(m), N, int(nnz), &one, descr, aVal, aEcsr, aVxl, e, &one, c);
      dividesMultiplies<val_t>(xx, x, c, s, N);
      CK(cudaMemcpy(x, xx, N * sizeof(float), cudaMemcpyDeviceToDevice));
      float nx = sum<val_t>(x, N);
      scales<val_t>(x, val_t(1. / nx), N);
    }
    CK(cudaMemcpy(hx.data(), x, N * sizeof(float), cudaMemcpyDeviceToHost));
    FILE* f = std::fopen(argv[1], "wb");
    std::fwrite(hx.data(), sizeof(float), N, f);
    std::fclose(f);
    std::printf("rows %u nnz %llu\n", m, nnz);
  } catch (const std::exception& ex) {
    std::fprintf(stderr, "error: %s\n", ex.what());
    return 1;
  }
  return 0;
}
