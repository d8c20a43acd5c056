// lbm_main.cpp — C++ driver with the behaviour of the reference main.cpp,
// written against the reference's own host spelling (lbm_b200_compat.hpp):
// build the case of main.cpp:59-85, report the tile decomposition
// (decomposition(), main.cpp:256-261), run the Initialize program and
// maxitr steps on the GPU timed with std::chrono around the run
// (main.cpp:308-314), read arF back (main.cpp:317) and print direction 9 of
// the plane k=2 (main.cpp:321-347).
//
//   lbm_main [h] [maxitr] [Cs] [srt|mrt] [nwrite] [savetype]
// Defaults are main.cpp's: h=10, maxitr=199, MRT+LES, Re=1000, u_lid=0.1,
// Smagorinsky constant 0 (main.cpp never assigns it), no result files.
// The steps run through runSimulation(Inputval*, LBMSolver*), kernel.cu's
// loop: a residual line every 100 cycles and, with nwrite > 0, a result
// file every nwrite cycles (savetype 0 = VTU, 1 = CSV, into ./result/).
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "../../include/lbm_b200_compat.hpp"

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
  in.casetype = CAVITY;
  in.m_dTau = 3.0f * in.m_dRefVelx * in.h / in.Re + 0.50f;
  in.dWeps = 3.0f;
  in.dWepsj = -5.5f;
  in.dWXX = -0.5f;

  static int Slice[TILE_NUM][DIMENSION][2];
  LBMSolver* psolver = new LBMSolver();
  int rc = 0;
  try {
    const int ntile = decomposition(&in, Slice);
    std::printf("Number of Tiles participating = %d\n", ntile);
    initialize(&in, psolver);  // the Initialize program (main.cpp:280-282)
    lbm_b200::check(lbm_sync(psolver->m_pDomain));
    const auto t0 = std::chrono::high_resolution_clock::now();
    std::printf(" - Running program\n");
    runSimulation(&in, psolver);  // Repeat(maxitr, runSimulation) (main.cpp:283-291)
    lbm_b200::check(lbm_sync(psolver->m_pDomain));
    const auto t1 = std::chrono::high_resolution_clock::now();
    const std::chrono::duration<double> el = t1 - t0;
    std::printf(" - Elapsed time(GPU) = %fs | h=%d | %.1f MLUPS\n", el.count(), in.h,
                (double)in.nx * in.ny * in.nz * in.maxitr / el.count() / 1e6);

    std::vector<float>& arF = psolver->m_HostNode.m_arF;  // engine.readTensor("D2H-arF")
    arF.resize((size_t)in.nx * in.ny * in.nz * DIRECTION_SIZE);
    lbm_b200::check(lbm_export_arF(psolver->m_pDomain, arF.data(), 0));
    std::printf("---------------------------------\n");
    const int k = in.nz > 2 ? 2 : 0;
    for (int j = in.ny - 1; j >= 0; j--) {
      for (int i = 0; i < in.nx; i++) {
        const size_t id =
            9 + DIRECTION_SIZE * ((size_t)i + (size_t)k * in.nx + (size_t)j * in.nx * in.nz);
        std::printf("%8.6f ", arF[id]);
      }
      std::printf("\n");
    }
    std::printf("\n---------------------------------\n");
  } catch (const lbm_b200::Error& e) {
    std::fprintf(stderr, " - Error: %s\n", e.what());
    rc = 1;
  }
  delete psolver;
  return rc;
}
