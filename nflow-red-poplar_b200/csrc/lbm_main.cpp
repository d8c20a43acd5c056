// lbm_main.cpp — C++ driver with the behaviour of the reference main.cpp:
// build the case of main.cpp:59-85, report the tile decomposition
// (main.cpp:256-261), initialise and run maxitr steps on the GPU timed with
// std::chrono around the run (main.cpp:308-314), read arF back
// (main.cpp:317) and print direction 9 of the plane k=2 (main.cpp:321-347).
//
//   lbm_main [h] [maxitr] [Cs] [srt|mrt] [nwrite] [savetype] [outdir]
// Defaults are main.cpp's: h=10, maxitr=199, MRT+LES, Re=1000, u_lid=0.1,
// Smagorinsky constant 0 (main.cpp never assigns it), no result files.
// With nwrite > 0 it also writes the result files of kernel.cu's loop
// (kernel.cu:203-228, savetype 0 = VTU, 1 = CSV, into outdir, default
// ./result/) every nwrite steps and prints kernel.cu's residual line every
// 100 steps (kernel.cu:232-248).  Each file is written by a host thread from
// a snapshot while the GPU keeps stepping.
#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <thread>
#include <vector>

#include "../../include/lbm_b200.h"

int main(int argc, char** argv) {
  Inputval in;
  std::memset(&in, 0, sizeof(in));
  in.h = argc > 1 ? std::atoi(argv[1]) : 10;
  in.nx = in.ny = in.nz = in.h;
  in.maxitr = argc > 2 ? std::atoi(argv[2]) : 199;
  in.m_dSmagorinsky = argc > 3 ? (float)std::atof(argv[3]) : 0.0f;
  const bool srt = argc > 4 && std::strcmp(argv[4], "srt") == 0;  // anything else: MRT+LES
  in.bEnableMRT = !srt;
  in.bEnableLES = !srt;
  in.m_dRefDen = 1.0f;
  in.m_dRefVelx = 0.1f;
  in.Re = 1000;
  in.length = (float)(in.nx * in.ny * in.nz);
  in.nu = in.m_dRefVelx * in.h / in.Re;
  in.nwrite = argc > 5 ? std::atoi(argv[5]) : 0;
  in.savetype = argc > 6 ? std::atoi(argv[6]) : 1;
  const char* outdir = argc > 7 ? argv[7] : nullptr;
  in.casetype = CAVITY;
  in.m_dTau = 3.0f * in.m_dRefVelx * in.h / in.Re + 0.50f;
  in.dWeps = 3.0f;
  in.dWepsj = -5.5f;
  in.dWXX = -0.5f;

  static int Slice[TILE_NUM][DIMENSION][2];
  int ntile = lbm_decomposition(&in, Slice);
  std::printf("Number of Tiles participating = %d\n", ntile);

  lbm_domain* d = nullptr;
  if (lbm_create(&in, nullptr, &d) != LBM_OK || lbm_initialize(d) != LBM_OK) {
    std::fprintf(stderr, " - Error: %s\n", lbm_last_error());
    if (d) lbm_destroy(d);
    return 1;
  }
  lbm_sync(d);
  auto t0 = std::chrono::high_resolution_clock::now();
  std::printf(" - Running program\n");
  bool ok = true;
  if (in.nwrite <= 0) {
    ok = lbm_run_simulation(d, in.maxitr) == LBM_OK && lbm_sync(d) == LBM_OK;
  } else {
    // kernel.cu's loop: a residual line every 100 steps, a file every nwrite
    std::thread writer;
    int write_rc = LBM_OK;
    for (int icycle = 0; ok && icycle < in.maxitr;) {
      const int next_print = (icycle / 100 + 1) * 100, next_write = (icycle / in.nwrite + 1) * in.nwrite;
      int k = std::min(std::min(next_print, next_write), in.maxitr) - icycle;
      ok = lbm_run_simulation(d, k) == LBM_OK;
      icycle += k;
      if (ok && icycle % 100 == 0) {
        double diag[8];
        ok = lbm_diagnostics(d, diag) == LBM_OK;
        if (ok) std::printf("ITER=%d | ERROR=%.5e\n", icycle, diag[4]);
      }
      if (ok && icycle % in.nwrite == 0) {
        if (writer.joinable()) writer.join();
        ok = write_rc == LBM_OK && lbm_snapshot(d) == LBM_OK;
        const int index = icycle / in.nwrite, type = in.savetype;
        if (ok) writer = std::thread([&write_rc, d, type, outdir, index] {
            write_rc = lbm_save_snapshot(d, type, outdir, index);
          });
      }
    }
    if (writer.joinable()) writer.join();
    ok = ok && write_rc == LBM_OK && lbm_sync(d) == LBM_OK;
  }
  if (!ok) {
    std::fprintf(stderr, " - Error: %s\n", lbm_last_error());
    lbm_destroy(d);
    return 1;
  }
  auto t1 = std::chrono::high_resolution_clock::now();
  std::chrono::duration<double> el = t1 - t0;
  std::printf(" - Elapsed time(GPU) = %fs | h=%d | %.1f MLUPS\n", el.count(), in.h,
              (double)in.nx * in.ny * in.nz * in.maxitr / el.count() / 1e6);

  std::vector<float> arF((size_t)in.nx * in.ny * in.nz * DIRECTION_SIZE);
  if (lbm_export_arF(d, arF.data(), 0) != LBM_OK) {
    std::fprintf(stderr, " - Error: %s\n", lbm_last_error());
    lbm_destroy(d);
    return 1;
  }
  std::printf("---------------------------------\n");
  const int k = in.nz > 2 ? 2 : 0;
  for (int j = in.ny - 1; j >= 0; j--) {
    for (int i = 0; i < in.nx; i++) {
      size_t id = 9 + DIRECTION_SIZE * ((size_t)i + (size_t)k * in.nx + (size_t)j * in.nx * in.nz);
      std::printf("%8.6f ", arF[id]);
    }
    std::printf("\n");
  }
  std::printf("\n---------------------------------\n");
  lbm_destroy(d);
  return 0;
}
