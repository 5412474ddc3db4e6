// reco: MLEM reconstruction from a measurement file, with the argv of the
// reference's src/tests/reco.cu:53-90:
//   reco <measurement.h5> <output.h5> <rays> <sensitivity.h5> <iterations> <guess.h5>
// writes "<it>_<output>" after every iteration (src/tests/reco.cu:305-311;
// for an output path with a directory the prefix goes on its file name).
// The system matrix of the measured channels is built once and kept in
// device memory with its transpose; an iteration is the library's two-pass
// MLEM (raptr_mlem).  Geometry: see common.hpp.
#include "common.hpp"

#include <fstream>

int main(int argc, char** argv) {
  const char* help[] = {"filename of measurement", "filename of output", "number of rays",
                        "filename of sensitivity", "number reco iterations", "filename of density guess"};
  if (argc != 7) return drv::usage(help, 6, argc);
  try {
    const std::string fn(argv[1]), on(argv[2]), sfn(argv[4]), xfn(argv[6]);
    const int nrays = std::atoi(argv[3]), nIt = std::atoi(argv[5]);
    drv::Timer t;
    raptr_geom g{};
    drv::setup_from(fn, &g);
    drv::grid_from_density(sfn, &g);
    const int64_t N = int64_t(g.grid_n[0]) * g.grid_n[1] * g.grid_n[2];

    std::vector<int> yId;
    std::vector<float> yVal;
    int effM = 0;
    readHDF5_MeasVct(yId, yVal, effM, fn);
    std::printf("measured channels: %d\n", effM);

    std::vector<float> s = readHDF5_Density<float>(sfn);
    if (int64_t(s.size()) != N) throw raptr::Exception("sensitivity size does not match the grid");
    double S = 0.0;
    for (float v : s) S += v;
    std::printf("S: %g\n", S);

    std::vector<float> x;
    if (std::ifstream(xfn).good()) {
      std::printf("Will use density from file %s\n", xfn.c_str());
      x = readHDF5_Density<float>(xfn);
      if (int64_t(x.size()) != N) throw raptr::Exception("density guess size does not match the grid");
    } else {
      x.assign(size_t(N), 1.f);
    }

    drv::Rows A;
    drv::build_rows(g, yId, nrays, &A);
    raptr::check(raptr_matrix_transpose(A.A, nullptr), "raptr_matrix_transpose");
    std::printf("system matrix: %lld rows, %lld entries (%.1f ms)\n", (long long)A.m, (long long)A.nnz, t.ms());

    int64_t *rp, *cp;
    int32_t *col, *ri, *order, *rank;
    float *val, *tv;
    raptr::check(raptr_matrix_info(A.A, nullptr, nullptr, nullptr, &rp, &col, &val), "raptr_matrix_info");
    raptr::check(raptr_matrix_csc_info(A.A, &cp, &ri, &tv), "raptr_matrix_csc_info");
    raptr::check(raptr_matrix_row_order(A.A, &order, &rank), "raptr_matrix_row_order");

    raptr::DeviceBuffer<float> d_y{static_cast<size_t>(effM)}, d_s{static_cast<size_t>(N)}, d_x{static_cast<size_t>(N)};
    raptr::check_cuda(cudaMemcpy(d_y.p, yVal.data(), size_t(effM) * 4, cudaMemcpyHostToDevice), "cudaMemcpy");
    raptr::check_cuda(cudaMemcpy(d_s.p, s.data(), size_t(N) * 4, cudaMemcpyHostToDevice), "cudaMemcpy");
    raptr::check_cuda(cudaMemcpy(d_x.p, x.data(), size_t(N) * 4, cudaMemcpyHostToDevice), "cudaMemcpy");
    // normalise the sensitivity (src/tests/reco.cu:202-204)
    const float norm = sum<float>(d_s.p, int(N));
    scales<float>(d_s.p, float(1. / norm), int(N));

    DefaultVoxelGrid<float> grid = drv::voxel_grid(g);
    raptr_mlem_opts o = {0, nullptr, nullptr, rank};
    for (int it = 0; it < nIt; it++) {
      drv::Timer ti;
      raptr::check(raptr_mlem(A.ctx, A.m, N, rp, col, val, cp, ri, tv, d_y.p, d_s.p, d_x.p, 1, &o, nullptr),
                   "raptr_mlem");
      raptr::check_cuda(cudaMemcpy(x.data(), d_x.p, size_t(N) * 4, cudaMemcpyDeviceToHost), "cudaMemcpy");
      // "<it>_<output>" (the iteration number prefixes the file name, in
      // the output's directory)
      const size_t slash = on.find_last_of('/');
      const std::string dir = slash == std::string::npos ? "" : on.substr(0, slash + 1);
      const std::string base = slash == std::string::npos ? on : on.substr(slash + 1);
      writeHDF5_Density(x.data(), dir + std::to_string(it) + "_" + base, grid);
      std::printf("iteration %d: %.2f ms\n", it, ti.ms());
    }
    std::printf("total: %.1f ms\n", t.ms());
  } catch (const std::exception& e) {
    std::fprintf(stderr, "reco: %s\n", e.what());
    return EXIT_FAILURE;
  }
  return 0;
}
