// pureSMCalculation: builds the system matrix of the measured channels and
// reports its size and build time, with the argv of
// src/tests/pureSMCalculation.cu:48-72:
//   pureSMCalculation <measurement.h5> <rays>
// Geometry: see common.hpp (the grid from RAPTR_GRID).
#include "common.hpp"

int main(int argc, char** argv) {
  const char* help[] = {"filename of measurement", "number of rays"};
  if (argc != 3) return drv::usage(help, 2, argc);
  try {
    const std::string fn(argv[1]);
    const int nrays = std::atoi(argv[2]);
    raptr_geom g{};
    drv::setup_from(fn, &g);
    drv::grid_from_env(&g);
    std::vector<int> yId;
    std::vector<float> yVal;
    int effM = 0;
    readHDF5_MeasVct(yId, yVal, effM, fn);
    drv::Timer t;
    drv::Rows A;
    drv::build_rows(g, yId, nrays, &A);
    raptr::check_cuda(cudaDeviceSynchronize(), "cudaDeviceSynchronize");
    const double ms = t.ms();
    std::printf("channels %d, entries %lld, build %.1f ms, %.3g rays/s\n", effM, (long long)A.nnz, ms,
                double(effM) * nrays / (ms / 1e3));
  } catch (const std::exception& e) {
    std::fprintf(stderr, "pureSMCalculation: %s\n", e.what());
    return EXIT_FAILURE;
  }
  return 0;
}
