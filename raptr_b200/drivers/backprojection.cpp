// backprojection: the measurement projected back onto the grid, normalised
// to sum 1, with the argv of src/tests/backprojection.cu:47-72:
//   backprojection <measurement.h5> <output.h5> <rays>
// Geometry: see common.hpp (the grid from RAPTR_GRID).
#include "common.hpp"

int main(int argc, char** argv) {
  const char* help[] = {"filename of measurement", "filename of output", "number of rays"};
  if (argc != 4) return drv::usage(help, 3, argc);
  try {
    const std::string fn(argv[1]), on(argv[2]);
    const int nrays = std::atoi(argv[3]);
    drv::Timer t;
    raptr_geom g{};
    drv::setup_from(fn, &g);
    drv::grid_from_env(&g);
    const int64_t N = int64_t(g.grid_n[0]) * g.grid_n[1] * g.grid_n[2];
    std::vector<int> yId;
    std::vector<float> yVal;
    int effM = 0;
    readHDF5_MeasVct(yId, yVal, effM, fn);
    drv::Rows A;
    drv::build_rows(g, yId, nrays, &A);
    int64_t* rp;
    int32_t* col;
    float* val;
    raptr::check(raptr_matrix_info(A.A, nullptr, nullptr, nullptr, &rp, &col, &val), "raptr_matrix_info");
    raptr::DeviceBuffer<float> d_y{static_cast<size_t>(effM)}, d_x{static_cast<size_t>(N)};
    raptr::check_cuda(cudaMemcpy(d_y.p, yVal.data(), size_t(effM) * 4, cudaMemcpyHostToDevice), "cudaMemcpy");
    // x = A^T y (src/tests/backprojection.cu:155-158), then x /= sum(x)
    raptr::check(raptr_spmv(RAPTR_OP_T, A.m, N, rp, col, val, 1.f, d_y.p, 0.f, d_x.p, nullptr), "raptr_spmv");
    const float norm = sum<float>(d_x.p, int(N));
    std::printf("Norm: %g\n", norm);
    scales<float>(d_x.p, float(1. / norm), int(N));
    std::vector<float> x(static_cast<size_t>(N));
    raptr::check_cuda(cudaMemcpy(x.data(), d_x.p, size_t(N) * 4, cudaMemcpyDeviceToHost), "cudaMemcpy");
    DefaultVoxelGrid<float> grid = drv::voxel_grid(g);
    writeHDF5_Density(x.data(), on, grid);
    std::printf("rows %lld, entries %lld, total %.1f ms\n", (long long)A.m, (long long)A.nnz, t.ms());
  } catch (const std::exception& e) {
    std::fprintf(stderr, "backprojection: %s\n", e.what());
    return EXIT_FAILURE;
  }
  return 0;
}
