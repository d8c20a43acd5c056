// lbm_output.cpp — the result files of kernel.cu's saveFile
// (kernel.cu:699-1018), written from host arrays in the [ny][nz][nx] node
// order of CurrDen / CurrVel* / NodeType.
//
// VTU (BINARYTYPE): the same VTK XML document as kernel.cu — element order,
// names, attribute text, appended raw encoding with a UInt64 byte count in
// front of every block — with two deliberate differences:
//   * every Float64 block holds real doubles.  kernel.cu writes 8 bytes
//     starting at each 4-byte float (kernel.cu:867-869, 906-916), so its
//     Float64 values are the bytes of two neighbouring floats;
//   * the cell list holds the (nx-1)(ny-1)(nz-1) hexahedra only.  kernel.cu
//     sizes its index array for nx*ny*nz cells (kernel.cu:26-27) and leaves
//     the tail zero, so its trailing cells are degenerate.
// CSV (CSVTYPE): result.csv and section.csv with kernel.cu's printf formats
// ("%d, %d, %d, %lf, %lf, %lf, %lf" and "%d, %lf"), byte for byte.
// Formatting runs on several host threads; the output order is the node
// order.
#include <algorithm>
#include <cerrno>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "../../include/lbm_b200.h"
#include "lbm_internal.h"

using lbm::set_error;

namespace {

struct File {
  FILE* f = nullptr;
  explicit File(const char* path, const char* mode) : f(std::fopen(path, mode)) {}
  ~File() {
    if (f) std::fclose(f);
  }
  bool write(const void* p, size_t n) { return std::fwrite(p, 1, n, f) == n; }
  bool puts(const std::string& s) { return write(s.data(), s.size()); }
  bool close() {
    const bool ok = std::fclose(f) == 0;
    f = nullptr;
    return ok;
  }
};

int io_error(const char* what, const char* path) {
  return set_error(LBM_ERR_IO, "%s %s: %s", what, path ? path : "(null)", std::strerror(errno));
}

// Appended block: UInt64 byte count, then the values produced by fill(i0, i1,
// buffer) for element ranges, in chunks so that memory stays bounded.
template <class T, class Fill>
bool put_block(File& out, uint64_t count, int per_elem, Fill&& fill) {
  const uint64_t bytes = count * per_elem * sizeof(T);
  if (!out.write(&bytes, sizeof(bytes))) return false;
  const uint64_t chunk = 1 << 20;
  std::vector<T> buf;
  for (uint64_t i0 = 0; i0 < count; i0 += chunk) {
    const uint64_t i1 = std::min(count, i0 + chunk);
    buf.resize((i1 - i0) * per_elem);
    fill(i0, i1, buf.data());
    if (!out.write(buf.data(), buf.size() * sizeof(T))) return false;
  }
  return true;
}

// Format nodes [0, n) with line(i, char*) -> length, on several threads,
// writing the text in node order.
template <class Line>
bool put_lines(File& out, long long n, size_t max_line, Line&& line) {
  const long long chunk = 1 << 16;
  const unsigned nthreads = std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
  std::vector<std::string> bufs(nthreads);
  for (long long base = 0; base < n; base += chunk * nthreads) {
    std::vector<std::thread> pool;
    for (unsigned t = 0; t < nthreads; ++t) {
      pool.emplace_back([&, t] {
        const long long i0 = base + (long long)t * chunk, i1 = std::min(n, i0 + chunk);
        std::string& b = bufs[t];
        b.clear();
        if (i0 >= i1) return;
        b.resize((size_t)(i1 - i0) * max_line);
        size_t len = 0;
        for (long long i = i0; i < i1; ++i) len += line(i, &b[len]);
        b.resize(len);
      });
    }
    for (auto& th : pool) th.join();
    for (unsigned t = 0; t < nthreads; ++t)
      if (!out.puts(bufs[t])) return false;
  }
  return true;
}

}  // namespace

extern "C" {

int lbm_write_vtu(const char* path, int nx, int ny, int nz, const float* den, const float* velx,
                  const float* vely, const float* velz, const int* node_type) {
  if (!path || !den || !velx || !vely || !velz || !node_type)
    return set_error(LBM_ERR_INVALID, "lbm_write_vtu: NULL argument");
  if (nx < 2 || ny < 2 || nz < 2)
    return set_error(LBM_ERR_INVALID, "lbm_write_vtu: every extent must be >= 2");
  const uint64_t npts = (uint64_t)nx * ny * nz;
  const uint64_t ncells = (uint64_t)(nx - 1) * (ny - 1) * (nz - 1);
  if (npts > 0x7fffffffull) return set_error(LBM_ERR_INVALID, "lbm_write_vtu: too many points");
  File out(path, "wb");
  if (!out.f) return io_error("cannot open", path);

  // header: kernel.cu:733-851 (byte offsets of the appended blocks)
  const uint64_t H = 8;  // UInt64 block header
  const uint64_t b_pts = npts * 3 * 8, b_conn = ncells * 8 * 4, b_off = ncells * 4,
                 b_type = ncells, b_vec = npts * 3 * 8, b_sca = npts * 8, b_flag = npts * 4;
  uint64_t off = 0;
  std::string h;
  auto arr = [&](const char* head, uint64_t bytes) {
    h += head + std::to_string(off) + "\" format=\"appended\"/>\n";
    off += bytes + H;
  };
  h += "<VTKFile type=\"UnstructuredGrid\" version=\"1.0\" byte_order=\"LittleEndian\" "
       "header_type=\"UInt64\">\n";
  h += "<UnstructuredGrid>\n";
  h += "<Piece NumberOfPoints=\"" + std::to_string(npts) + "\" NumberOfCells=\"" +
       std::to_string(ncells) + "\">\n";
  h += "<Points>\n";
  arr("<DataArray type=\"Float64\" Name=\"\" NumberOfComponents=\"3\" offset=\"", b_pts);
  h += "</Points>\n<Cells>\n";
  arr("<DataArray type=\"Int32\" Name=\"connectivity\" NumberOfComponents= \"1\" offset=\"",
      b_conn);
  arr("<DataArray type=\"Int32\" Name=\"offsets\" NumberOfComponents= \"1\" offset=\"", b_off);
  arr("<DataArray type=\"UInt8\" Name=\"types\" NumberOfComponents= \"1\" offset=\"", b_type);
  h += "</Cells>\n<PointData>\n";
  arr("<DataArray type = \"Float64\" Name=\"Velocity\" NumberOfComponents= \"3\" offset=\"",
      b_vec);
  arr("<DataArray type = \"Float64\" Name=\"Density\" NumberOfComponents= \"1\" offset=\"",
      b_sca);
  static const char* kFlagNames[6] = {"Fluid", "Fixed Wall", "Moving Wall",
                                      "Inlet", "Outlet",     "Struct"};
  for (const char* name : kFlagNames)
    arr((std::string("<DataArray type = \"Int32\" Name=\"") + name +
         "\" NumberOfComponents= \"1\" offset=\"")
            .c_str(),
        b_flag);
  h += "</PointData>\n</Piece>\n</UnstructuredGrid>\n";
  h += "<AppendedData encoding=\"raw\">\n_";
  bool ok = out.puts(h);

  const uint64_t slave = (uint64_t)nx * nz;
  // points (x, y, z) of node i = x + nx*(z + nz*y)
  ok = ok && put_block<double>(out, npts, 3, [&](uint64_t i0, uint64_t i1, double* b) {
         for (uint64_t i = i0; i < i1; ++i, b += 3) {
           b[0] = (double)((i % slave) % nx);
           b[1] = (double)(i / slave);
           b[2] = (double)((i % slave) / nx);
         }
       });
  // connectivity: hexahedron at (x, y, z) < (nx-1, ny-1, nz-1), vertices
  // (x,z) (x+1,z) (x+1,z+1) (x,z+1) on plane y then plane y+1
  // (kernel.cu:29-57)
  const uint64_t cx = nx - 1, cz = nz - 1;
  ok = ok && put_block<int32_t>(out, ncells, 8, [&](uint64_t i0, uint64_t i1, int32_t* b) {
         for (uint64_t c = i0; c < i1; ++c, b += 8) {
           const uint64_t x = c % cx, z = (c / cx) % cz, y = c / (cx * cz);
           for (int k = 0; k < 2; ++k) {
             const uint64_t base = slave * (y + k);
             b[4 * k + 0] = (int32_t)(base + nx * z + x);
             b[4 * k + 1] = (int32_t)(base + nx * z + x + 1);
             b[4 * k + 2] = (int32_t)(base + nx * (z + 1) + x + 1);
             b[4 * k + 3] = (int32_t)(base + nx * (z + 1) + x);
           }
         }
       });
  ok = ok && put_block<int32_t>(out, ncells, 1, [&](uint64_t i0, uint64_t i1, int32_t* b) {
         for (uint64_t c = i0; c < i1; ++c) *b++ = (int32_t)(8 + c * 8);
       });
  ok = ok && put_block<uint8_t>(out, ncells, 1, [&](uint64_t i0, uint64_t i1, uint8_t* b) {
         std::memset(b, 12, i1 - i0);  // VTK_HEXAHEDRON
       });
  ok = ok && put_block<double>(out, npts, 3, [&](uint64_t i0, uint64_t i1, double* b) {
         for (uint64_t i = i0; i < i1; ++i, b += 3) {
           b[0] = velx[i];
           b[1] = vely[i];
           b[2] = velz[i];
         }
       });
  ok = ok && put_block<double>(out, npts, 1, [&](uint64_t i0, uint64_t i1, double* b) {
         for (uint64_t i = i0; i < i1; ++i) *b++ = den[i];
       });
  static const int kFlagBits[6] = {NODE_FLUID, NODE_FIXEDWALL, NODE_MOVINGWALL,
                                   NODE_INLET, NODE_OUTLET,    NODE_STRUCT};
  for (int bit : kFlagBits)
    ok = ok && put_block<int32_t>(out, npts, 1, [&](uint64_t i0, uint64_t i1, int32_t* b) {
           for (uint64_t i = i0; i < i1; ++i) *b++ = (node_type[i] & bit) ? 1 : 0;
         });
  ok = ok && out.puts("</AppendedData>\n</VTKFile>");
  if (!ok || !out.close()) return io_error("cannot write", path);
  return LBM_OK;
}

int lbm_write_csv(const char* result_path, const char* section_path, int nx, int ny, int nz,
                  const float* den, const float* velx, const float* vely, const float* velz) {
  if (!den || !velx || !vely || !velz)
    return set_error(LBM_ERR_INVALID, "lbm_write_csv: NULL field");
  if (nx < 1 || ny < 1 || nz < 1) return set_error(LBM_ERR_INVALID, "lbm_write_csv: bad extent");
  const long long n = (long long)nx * ny * nz, slave = (long long)nx * nz;
  if (result_path) {
    File out(result_path, "wt");
    if (!out.f) return io_error("cannot open", result_path);
    bool ok = out.puts("x,y,z,rho,u,v,w\n");
    // kernel.cu:987-996
    ok = ok && put_lines(out, n, 512, [&](long long i, char* p) -> size_t {
           const int x = (int)((i % slave) % nx), y = (int)(i / slave),
                     z = (int)((i % slave) / nx);
           return (size_t)std::snprintf(p, 512, "%d, %d, %d, %lf, %lf, %lf, %lf\n", x, y, z,
                                        (double)den[i], (double)velx[i], (double)vely[i],
                                        (double)velz[i]);
         });
    if (!ok || !out.close()) return io_error("cannot write", result_path);
  }
  if (section_path) {
    File out(section_path, "wt");
    if (!out.f) return io_error("cannot open", section_path);
    // kernel.cu:1002-1014: the line x = z = 49 (the pipe axis of the
    // POISEUILLE case), u_x scaled by 10
    std::string s = "y/Y,u\n";
    if (nx > 49 && nz > 49) {
      char line[128];
      for (int y = 0; y < ny; ++y) {
        const long long i = 49 + (long long)nx * (49 + (long long)nz * y);
        std::snprintf(line, sizeof(line), "%d, %lf\n", y, (double)(velx[i] * 10));
        s += line;
      }
    }
    if (!out.puts(s) || !out.close()) return io_error("cannot write", section_path);
  }
  return LBM_OK;
}

}  // extern "C"
