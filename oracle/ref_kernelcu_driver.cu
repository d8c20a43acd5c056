/*
 * ref_kernelcu_driver.cu — TEST INFRASTRUCTURE ONLY (the oracle's reference
 * leg for the parts that exist only in the legacy CUDA solver).
 *
 * Includes the reference's kernel.cu unmodified (built from the reference
 * tree by oracle/Makefile into oracle/_ref/libkernelcu_ref.so) and launches
 * its own __global__ kernels in the order of its host loop
 * (kernel.cu:154-199): LES -> MRT|SRT -> keStreaming -> boundary kernels ->
 * keMacroscopic.  Only the host side is this project's: device allocation,
 * the table uploads of kernel.cu:97-107 (Move is the unpadded offset table
 * that main.cpp:119-137 leaves commented out) and the initial state, which
 * is built on the host with the Initialize codelet's formula so that the
 * seeded perturbations of orc_common.h can be applied.
 *
 * Runs on a CUDA GPU only.  Used by the gpu tests to pin the oracle port's
 * SRT / inlet / outlet / struct restatement against the reference itself and
 * to generate tests/golden/kernelcu_*.npz.
 */
#include <sys/stat.h>
#include <unistd.h>

#include <string>
#include <vector>

#include "struct.h"
#include "kernel.cu" /* reference */

#include "orc_common.h"

/* main.cpp:29-33 defines LBMSolver's constructor and destructor empty;
 * main.cpp is not built here, so the driver supplies the same. */
LBMSolver::LBMSolver() {}
LBMSolver::~LBMSolver() {}

namespace {
const int kCx[19] = {0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, 0, 0, 0, 0};
const int kCy[19] = {0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, 1, -1, -1, 1, 1, -1, -1};
const int kCz[19] = {0, 0, 0, -1, 1, 0, 0, -1, -1, 1, 1, 0, 0, 0, 0, -1, 1, -1, 1};
const int kOpp[19] = {0, 2, 1, 4, 3, 6, 5, 10, 9, 8, 7, 14, 13, 12, 11, 18, 17, 16, 15};
const float kM[19][19] = {
    {1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1},
    {-30, -11, -11, -11, -11, -11, -11, 8, 8, 8, 8, 8, 8, 8, 8, 8, 8, 8, 8},
    {12, -4, -4, -4, -4, -4, -4, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1},
    {0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, 0, 0, 0, 0},
    {0, -4, 4, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, 0, 0, 0, 0},
    {0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, 1, -1, -1, 1, 1, -1, -1},
    {0, 0, 0, 0, 0, -4, 4, 0, 0, 0, 0, 1, 1, -1, -1, 1, 1, -1, -1},
    {0, 0, 0, -1, 1, 0, 0, -1, -1, 1, 1, 0, 0, 0, 0, -1, 1, -1, 1},
    {0, 0, 0, 4, -4, 0, 0, -1, -1, 1, 1, 0, 0, 0, 0, -1, 1, -1, 1},
    {0, 2, 2, -1, -1, -1, -1, 1, 1, 1, 1, 1, 1, 1, 1, -2, -2, -2, -2},
    {0, -4, -4, 2, 2, 2, 2, 1, 1, 1, 1, 1, 1, 1, 1, -2, -2, -2, -2},
    {0, 0, 0, -1, -1, 1, 1, -1, -1, -1, -1, 1, 1, 1, 1, 0, 0, 0, 0},
    {0, 0, 0, 2, 2, -2, -2, -1, -1, -1, -1, 1, 1, 1, 1, 0, 0, 0, 0},
    {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 1, -1, -1, 1, 0, 0, 0, 0},
    {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, -1, 1, 1, -1},
    {0, 0, 0, 0, 0, 0, 0, -1, 1, 1, -1, 0, 0, 0, 0, 0, 0, 0, 0},
    {0, 0, 0, 0, 0, 0, 0, -1, 1, -1, 1, 1, -1, 1, -1, 0, 0, 0, 0},
    {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, -1, -1, 1, 1, 1, 1, -1, -1},
    {0, 0, 0, 0, 0, 0, 0, -1, -1, 1, 1, 0, 0, 0, 0, 1, -1, 1, -1}};

int node_type_host(const Inputval* in, int x, int y, int z) {
  int t = NODE_FLUID;
  if (in->casetype == CAVITY) {
    if (y == 0) t = NODE_FIXEDWALL;
    if (y == in->ny - 1) t = NODE_MOVINGWALL;
    if (x == 0 || x == in->nx - 1 || z == 0 || z == in->nz - 1) t = NODE_FIXEDWALL;
  } else if (in->casetype == POISEUILLE) {
    if (x == 0) t = NODE_INLET;
    if (x == in->nx - 1) t = NODE_OUTLET;
    if ((y - 25) * (y - 25) + (z - 25) * (z - 25) > 400) t = NODE_STRUCT;
  }
  return t;
}
}  // namespace

extern "C" {

/* Run the reference kernels for nsteps steps (after the initial state).
 * Outputs: arF AoS [ny][nz][nx][19] (post-stream, post-boundary),
 * den/ux/uy/uz [ny][nz][nx] (CurrDen/CurrVel), any may be NULL.
 * Returns 0, or the CUDA error code. */
int kref_run_solid(const Inputval* pin, const orc_ext* ext, int nsteps,
                   const unsigned char* solid, float* arF, float* den, float* ux, float* uy,
                   float* uz);

int kref_run(const Inputval* pin, const orc_ext* ext, int nsteps, float* arF, float* den,
             float* ux, float* uy, float* uz) {
  return kref_run_solid(pin, ext, nsteps, nullptr, arF, den, ux, uy, uz);
}

/* kref_run with solid voxels: nodes with solid[n] != 0 ([ny][nz][nx]) are
 * made NODE_STRUCT in the NodeType array the reference kernels read (the
 * geometry of keSetNodeType otherwise), so that the reference's own
 * keStreaming / keBoundaryStruct run on arbitrary obstacles.  The
 * reference applies keBoundaryStruct in the POISEUILLE case only
 * (kernel.cu:202-212), so only that case is comparable. */
int kref_run_solid(const Inputval* pin, const orc_ext* ext, int nsteps,
                   const unsigned char* solid, float* arF, float* den, float* ux, float* uy,
                   float* uz) {
  Inputval in = *pin;
  const int nx = in.nx, ny = in.ny, nz = in.nz;
  const int N = nx * ny * nz;
  const int nSlave = nx * nz;
  float hDir[DIMENSION * DIRECTION_SIZE], hW[DIRECTION_SIZE];
  int hOpp[DIRECTION_SIZE], hMove[DIRECTION_SIZE];
  for (int d = 0; d < 19; ++d) {
    hDir[XDIM * 19 + d] = (float)kCx[d];
    hDir[YDIM * 19 + d] = (float)kCy[d];
    hDir[ZDIM * 19 + d] = (float)kCz[d];
    hW[d] = d == 0 ? 1.0f / 3.0f : (d < 7 ? 1.0f / 18.0f : 1.0f / 36.0f);
    hOpp[d] = kOpp[d];
    hMove[d] = kCx[d] + kCz[d] * nx + kCy[d] * nSlave;
  }
  std::vector<std::vector<float>> mat(19, std::vector<float>(19));
  std::vector<std::vector<float>> inv(19, std::vector<float>(19, 0.0f));
  for (int i = 0; i < 19; ++i)
    for (int j = 0; j < 19; ++j) mat[i][j] = kM[i][j];
  inverseMRT(mat, inv); /* reference */
  MRTMatrix hMat;
  for (int i = 0; i < 19; ++i)
    for (int j = 0; j < 19; ++j) {
      hMat.m_MatMRT[i][j] = mat[i][j];
      hMat.m_MatInv[i][j] = inv[i][j];
    }

  /* initial state on the host: Initialize codelet formula + perturbation */
  std::vector<float> f0((size_t)N * 19, 0.0f), d0(N, 0.0f), x0(N, 0.0f), y0(N, 0.0f),
      z0(N, 0.0f);
  std::vector<int> t0(N);
  for (int y = 0; y < ny; ++y)
    for (int z = 0; z < nz; ++z)
      for (int x = 0; x < nx; ++x) {
        const int n = x + z * nx + y * nSlave;
        const int t = (solid && solid[n]) ? NODE_STRUCT : node_type_host(&in, x, y, z);
        t0[n] = t;
        if (t == NODE_STRUCT) continue;
        float dn = in.m_dRefDen, vx = 0.f, vy = 0.f, vz = 0.f;
        if (t == NODE_MOVINGWALL) {
          vx = in.m_dRefVelx;
          vy = in.m_dRefVely;
          vz = in.m_dRefVelz;
        }
        if (ext && ext->init_kind == 1)
          dn = (float)((double)in.m_dRefDen +
                       (double)ext->noise_amp * orc_unit_noise(ext->seed, (uint64_t)n, 0));
        for (int d = 0; d < 19; ++d) {
          float eu = hDir[XDIM * 19 + d] * vx + hDir[YDIM * 19 + d] * vy + hDir[ZDIM * 19 + d] * vz;
          float usq = vx * vx + vy * vy + vz * vz;
          f0[(size_t)d * N + n] = hW[d] * dn * (1.0f + 3.0f * eu + 4.5f * eu * eu - 1.5f * usq);
        }
        d0[n] = dn;
        x0[n] = vx;
        y0[n] = vy;
        z0[n] = vz;
      }

  float *dDir, *dW, *dF, *dFT, *dDen, *dPDen, *dVx, *dVy, *dVz, *dTau;
  int *dOpp, *dMove, *dType, *dDS;
  MRTMatrix* dMat;
  cudaError_t e = cudaSuccess;
#define KR(call)                     \
  do {                               \
    e = (call);                      \
    if (e != cudaSuccess) return (int)e; \
  } while (0)
  KR(cudaMalloc(&dMat, sizeof(MRTMatrix)));
  KR(cudaMalloc(&dDir, sizeof(hDir)));
  KR(cudaMalloc(&dW, sizeof(hW)));
  KR(cudaMalloc(&dOpp, sizeof(hOpp)));
  KR(cudaMalloc(&dMove, sizeof(hMove)));
  KR(cudaMalloc(&dF, sizeof(float) * N * 19));
  KR(cudaMalloc(&dFT, sizeof(float) * N * 19));
  KR(cudaMalloc(&dDen, sizeof(float) * N));
  KR(cudaMalloc(&dPDen, sizeof(float) * N));
  KR(cudaMalloc(&dVx, sizeof(float) * N));
  KR(cudaMalloc(&dVy, sizeof(float) * N));
  KR(cudaMalloc(&dVz, sizeof(float) * N));
  KR(cudaMalloc(&dTau, sizeof(float) * N));
  KR(cudaMalloc(&dType, sizeof(int) * N));
  KR(cudaMalloc(&dDS, sizeof(int) * N));
  KR(cudaMemcpy(dMat, &hMat, sizeof(MRTMatrix), cudaMemcpyHostToDevice));
  KR(cudaMemcpy(dDir, hDir, sizeof(hDir), cudaMemcpyHostToDevice));
  KR(cudaMemcpy(dW, hW, sizeof(hW), cudaMemcpyHostToDevice));
  KR(cudaMemcpy(dOpp, hOpp, sizeof(hOpp), cudaMemcpyHostToDevice));
  KR(cudaMemcpy(dMove, hMove, sizeof(hMove), cudaMemcpyHostToDevice));
  KR(cudaMemset(dFT, 0, sizeof(float) * N * 19));
  KR(cudaMemset(dTau, 0, sizeof(float) * N));
  KR(cudaMemset(dPDen, 0, sizeof(float) * N));

  const int blockSize = 512;
  const int gridSize = (N + blockSize - 1) / blockSize;
  int3 nNodeSize = {nx, ny, nz};
  keInitialNodeDirection<<<gridSize, blockSize>>>(dDS, nNodeSize, dDir, N);
  keSetNodeType<<<gridSize, blockSize>>>(dType, nNodeSize, N, in.casetype);
  KR(cudaGetLastError());
  if (solid) KR(cudaMemcpy(dType, t0.data(), sizeof(int) * N, cudaMemcpyHostToDevice));
  KR(cudaMemcpy(dF, f0.data(), sizeof(float) * N * 19, cudaMemcpyHostToDevice));
  KR(cudaMemcpy(dDen, d0.data(), sizeof(float) * N, cudaMemcpyHostToDevice));
  KR(cudaMemcpy(dVx, x0.data(), sizeof(float) * N, cudaMemcpyHostToDevice));
  KR(cudaMemcpy(dVy, y0.data(), sizeof(float) * N, cudaMemcpyHostToDevice));
  KR(cudaMemcpy(dVz, z0.data(), sizeof(float) * N, cudaMemcpyHostToDevice));

  for (int it = 0; it < nsteps; ++it) {
    if (in.bEnableLES)
      keComputeTurbulence_LES<<<gridSize, blockSize>>>(dType, dDen, dVx, dVy, dVz, dTau, dF, dW,
                                                       dDir, in.m_dTau, in.m_dSmagorinsky, N);
    if (in.bEnableMRT)
      keCollision_MRT<<<gridSize, blockSize>>>(dType, dDen, dVx, dVy, dVz, dTau, dF, dFT,
                                               in.m_dRefDen, in.m_dTau, in.dWeps, in.dWepsj,
                                               in.dWXX, dMat, N);
    else
      keCollision_SRT<<<gridSize, blockSize>>>(dType, dDen, dVx, dVy, dVz, dF, dFT, dW, dDir,
                                               in.m_dTau, dTau, N);
    keStreaming<<<gridSize, blockSize>>>(dType, dF, dFT, dDS, dMove, N);
    if (in.casetype == CAVITY) {
      keBoundaryCavity<<<gridSize, blockSize>>>(nNodeSize, dType, in.m_dRefVelx, in.m_dRefVely,
                                                in.m_dRefVelz, dF, dFT, dW, dDir, dDS, dOpp,
                                                in.m_dRefDen, N);
    } else if (in.casetype == POISEUILLE) {
      keBoundaryStruct<<<gridSize, blockSize>>>(nNodeSize, dType, dF, dFT, dDS, dOpp, dMove, N);
      keBoundaryInlet<<<gridSize, blockSize>>>(nNodeSize, dDen, dType, in.m_dRefVelx,
                                               in.m_dRefVely, in.m_dRefVelz, dF, dFT, dW, dDir,
                                               dDS, dOpp, dMove, N);
      keBoundaryOutlet<<<gridSize, blockSize>>>(nNodeSize, dVx, dVy, dVz, dType, dF, dFT, dW,
                                                dDir, dDS, dOpp, in.m_dRefDen, dMove, N);
    }
    keMacroscopic<<<gridSize, blockSize>>>(dType, dDen, dPDen, dVx, dVy, dVz, dF, dDir, N);
    KR(cudaGetLastError());
  }
  KR(cudaDeviceSynchronize());
  if (arF) {
    std::vector<float> soa((size_t)N * 19);
    KR(cudaMemcpy(soa.data(), dF, sizeof(float) * N * 19, cudaMemcpyDeviceToHost));
    for (int n = 0; n < N; ++n)
      for (int d = 0; d < 19; ++d) arF[(size_t)n * 19 + d] = soa[(size_t)d * N + n];
  }
  if (den) KR(cudaMemcpy(den, dDen, sizeof(float) * N, cudaMemcpyDeviceToHost));
  if (ux) KR(cudaMemcpy(ux, dVx, sizeof(float) * N, cudaMemcpyDeviceToHost));
  if (uy) KR(cudaMemcpy(uy, dVy, sizeof(float) * N, cudaMemcpyDeviceToHost));
  if (uz) KR(cudaMemcpy(uz, dVz, sizeof(float) * N, cudaMemcpyDeviceToHost));
  cudaFree(dMat);
  cudaFree(dDir);
  cudaFree(dW);
  cudaFree(dOpp);
  cudaFree(dMove);
  cudaFree(dF);
  cudaFree(dFT);
  cudaFree(dDen);
  cudaFree(dPDen);
  cudaFree(dVx);
  cudaFree(dVy);
  cudaFree(dVz);
  cudaFree(dTau);
  cudaFree(dType);
  cudaFree(dDS);
  return 0;
#undef KR
}

/* The reference's saveFile (kernel.cu:699-1018) on host fields
 * [ny][nz][nx]: writes result.csv + section.csv (savetype CSVTYPE) or
 * result/Output%06d.vtu (BINARYTYPE, index = file number) into workdir.
 * The cell index array is built as kernel.cu:26-57 builds it inside
 * runSimulation.  Host code only: needs no GPU.  Returns 0, or -1 when
 * workdir is not usable. */
int kref_save_file(const Inputval* pin, const float* den, const float* ux, const float* uy,
                   const float* uz, const int* ntype, int savetype, int index,
                   const char* workdir) {
  Inputval in = *pin;
  const int nx = in.nx, ny = in.ny, nz = in.nz;
  const int N = nx * ny * nz;
  in.length = (float)N;
  in.irestart = 0;
  in.nwrite = 1;
  in.icycle = index;
  LBMSolver* ps = new LBMSolver();
  HostNodeData& h = ps->m_HostNode;
  /* saveFile reads 8 bytes from every 4-byte value of these arrays
   * (kernel.cu:906-916); one spare element keeps the last read inside the
   * allocation */
  for (std::vector<float>* v : {&h.m_dCurrDen, &h.m_dCurrVelx, &h.m_dCurrVely, &h.m_dCurrVelz})
    v->reserve(N + 2);
  h.m_dCurrDen.assign(den, den + N);
  h.m_dCurrVelx.assign(ux, ux + N);
  h.m_dCurrVely.assign(uy, uy + N);
  h.m_dCurrVelz.assign(uz, uz + N);
  h.m_nNodeType.assign(ntype, ntype + N);
  std::vector<int> arIndex((size_t)N * 8, 0);
  int k = 0;
  for (int n = 0; n < N; ++n) {
    const int slave = nx * nz, x = (n % slave) % nx, y = n / slave, z = (n % slave) / nx;
    if (x >= nx - 1 || y >= ny - 1 || z >= nz - 1) continue;
    for (int y2 = y; y2 < y + 2; ++y2)
      for (int c = 0; c < 4; ++c) {
        const int x2 = x + (c == 1 || c == 2), z2 = z + (c >= 2);
        arIndex[k++] = nz * nx * y2 + nx * z2 + x2;
      }
  }
  char cwd[4096];
  if (!getcwd(cwd, sizeof(cwd)) || chdir(workdir) != 0) {
    delete ps;
    return -1;
  }
  mkdir("result", 0755); /* SAVE_PATH: saveFile exits when it cannot open the file */
  saveFile(&in, ps, arIndex, savetype); /* reference */
  const int rc = chdir(cwd) == 0 ? 0 : -1;
  delete ps;
  return rc;
}

}  // extern "C"
