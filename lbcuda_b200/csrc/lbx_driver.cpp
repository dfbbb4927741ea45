// lbx_driver.cpp — command-line host of the hot path (the role of LBcuda's
// `program TestLB`, main.CUF:1-316) written against the C ABI only.
//
//   lbx_run [options] [input.dat]
//     -L n | --nx n --ny n --nz n   lattice (the reference's MYDIMESION)
//     --storage f32|f16|bf16|f64|f16sd|bf16sd    population storage
//     --bgk                         single-component BGK instead of CG
//     --sigma s --beta b --tauR t --tauB t --tau t
//     --radius r --rmass m --neutral (wetting) --xyz file
//     --out dir                     VTI/VTK output directory (default output)
//     --seed s                      seed of initType 6
//     --restart-out dir             after the last step, write the restart
//                                   files of initType 4 (rhoR/rhoB.init.bin,
//                                   popR/popB.NNNNNN.init.bin) into dir
//
// initType 3 reads rhoR.init.bin / rhoB.init.bin and initType 4 also the
// per-direction population files popR/popB.NNNNNN.init.bin (read_and_setPops,
// main.CUF:2444-2529) from the working directory.
//
// input.dat is read with the rules of readParameters (main.CUF:409-496);
// input.xyz with those of read_input_atom (main.CUF:1230-1350).  Every
// nIterOut steps it prints Mlup/s (interior cells; the reference counts the
// halo too, (glx+2)^3, main.CUF:288) and every nIterVTK steps it writes
// rho/velocity/phase as VTK image data (writeImageDataVTI,
// write_output.f90:115-392) and the spheres as legacy VTK
// (writeParticleVTK, write_output.f90:674-746).
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <random>
#include <sstream>
#include <string>
#include <sys/stat.h>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/lbx.h"

namespace {

struct Deck {
  int nIter = 5, nIterOut = 1, nIterVTK = 100000000, initType = -1;
  float vx = 0, vy = 0, vz = 0;
  bool withParticles = false, lrotate = false;
  int numAtoms = 1;
  float ext_f[3] = {0, 0, 0}, ext_t[3] = {0, 0, 0};
  float max_vel = 0;
};

std::vector<std::string> tokens_of(const std::string& line) {
  std::string s = line.substr(0, line.find('!'));
  std::istringstream is(s);
  std::vector<std::string> t;
  std::string w;
  while (is >> w) t.push_back(w);
  return t;
}

// readParameters (main.CUF:409-496); returns false with the reference's
// messages on a short deck
bool read_deck(const char* path, Deck& d) {
  std::ifstream in(path);
  if (!in) {
    std::fprintf(stderr, "input.dat] Error opening file. STOP\n");
    return false;
  }
  std::vector<std::vector<std::string>> L;
  std::string line;
  while (std::getline(in, line)) {
    auto t = tokens_of(line);
    if (!t.empty()) L.push_back(t);
  }
  int found = 0, max_vel_found = 0;
  size_t i = 0;
  auto ok_int = [](const std::string& s, int& v) {
    char* e;
    long x = std::strtol(s.c_str(), &e, 10);
    if (*e) return false;
    v = int(x);
    return true;
  };
  do {
    if (i >= L.size() || !ok_int(L[i][0], d.nIter)) break;
    found = 1; ++i;
    if (i >= L.size() || !ok_int(L[i][0], d.nIterOut)) break;
    found = 2; ++i;
    if (i >= L.size() || !ok_int(L[i][0], d.nIterVTK)) break;
    found = 3; ++i;
    if (i >= L.size() || !ok_int(L[i][0], d.initType)) break;
    found = 4; ++i;
    if (i >= L.size() || L[i].size() < 3) break;
    d.vx = std::stof(L[i][0]); d.vy = std::stof(L[i][1]); d.vz = std::stof(L[i][2]);
    found = 5; ++i;
    if (i >= L.size()) break;
    if (L[i].size() > 1) d.numAtoms = std::atoi(L[i][1].c_str());
    found = 6;
    if (L[i][0].rfind("YES", 0) == 0) d.withParticles = true;
    else if (L[i][0].rfind("NO", 0) == 0) d.withParticles = false;
    else found = 5;
    ++i;
    if (!d.withParticles) break;
    if (i >= L.size() || L[i].size() < 3) break;
    for (int k = 0; k < 3; ++k) d.ext_f[k] = std::stof(L[i][k]);
    found = 7; ++i;
    if (i >= L.size()) break;
    if (L[i].size() > 1) d.max_vel = std::stof(L[i][1]);
    found = 8;
    found = 7;  // string(1:3) == 'MAX_PARTICLE_VEL' never holds (main.CUF:457-462)
    ++i;
    if (i >= L.size()) break;
    found = 9;
    if (L[i][0].rfind("YES", 0) == 0) d.lrotate = true;
    else if (L[i][0].rfind("NO", 0) == 0) d.lrotate = false;
    else found = 8;
    ++i;
    if (!d.lrotate) break;
    if (i >= L.size() || L[i].size() < 3) break;
    for (int k = 0; k < 3; ++k) d.ext_t[k] = std::stof(L[i][k]);
    found = 10;
  } while (false);
  bool bad = (d.lrotate && found != 10) || (!d.lrotate && d.withParticles && found != 9) ||
             (!d.withParticles && found != 6);
  if (bad) {
    if (found < 1) std::fprintf(stderr, "Number of iterations not found\n");
    if (found < 2) std::fprintf(stderr, "nIterOut not found\n");
    if (found < 3) std::fprintf(stderr, "nIterVTK not found\n");
    if (found < 4) std::fprintf(stderr, "initType not found\n");
    if (found < 5) std::fprintf(stderr, "vx,vy,vz,densR,densB not found\n");
    if (found < 6) std::fprintf(stderr, "withParticles not found\n");
    if (d.withParticles && found < 7) std::fprintf(stderr, "ext_fxx,ext_fyy,ext_fzz not found\n");
    if (d.withParticles && max_vel_found < 1) std::fprintf(stderr, "MAX_PARTICLE_VEL not found\n");
    if (d.withParticles && found < 9) std::fprintf(stderr, "lrotate not found\n");
    if (d.lrotate && found < 10) std::fprintf(stderr, "ext_tqx,ext_tqy,ext_tqz not found\n");
  }
  return !bad;
}

// eul2q (main.CUF:1352-1370)
void eul2q(float phis, float psis, float thetas, double q[4]) {
  float cy = std::cos(phis * 0.5f), sy = std::sin(phis * 0.5f);
  float cp = std::cos(psis * 0.5f), sp = std::sin(psis * 0.5f);
  float cr = std::cos(thetas * 0.5f), sr = std::sin(thetas * 0.5f);
  q[0] = cy * cp * cr + sy * sp * sr;
  q[1] = cy * cp * sr - sy * sp * cr;
  q[2] = sy * cp * sr + cy * sp * cr;
  q[3] = sy * cp * cr - cy * sp * sr;
}

bool read_xyz(const char* path, int n, bool lrotate, std::vector<double>& x, std::vector<double>& v,
              std::vector<double>& q) {
  std::ifstream in(path);
  if (!in) {
    std::fprintf(stderr, "input.xyz] Error opening file. STOP\n");
    return false;
  }
  std::string line;
  std::getline(in, line);
  int nf = std::atoi(line.c_str());
  if (nf < n) {
    std::fprintf(stderr, "Input file:input.xyz contains less particles than needed. STOP\n");
    return false;
  }
  std::getline(in, line);
  x.assign(3 * size_t(n), 0);
  v.assign(3 * size_t(n), 0);
  q.assign(4 * size_t(n), 0);
  for (int a = 0; a < n; ++a) {
    std::getline(in, line);
    std::istringstream is(line);
    std::string tag;
    double e[3] = {0, 0, 0};
    is >> tag >> x[3 * a] >> x[3 * a + 1] >> x[3 * a + 2] >> v[3 * a] >> v[3 * a + 1] >> v[3 * a + 2];
    q[4 * a] = 1.0;
    if (lrotate) {
      is >> e[0] >> e[1] >> e[2];
      eul2q(float(e[0]), float(e[2]), float(e[1]), &q[4 * a]);
    }
  }
  return true;
}

float fcut(float r, float r1, float r2) {  // kernels_fluid_CG.CUF:126-138
  if (r <= r1) return 1.0f;
  if (r > r2) return 0.0f;
  return 0.5f * std::cos((r - r1) * 3.14159265358979f / (r2 - r1)) + 0.5f;
}

bool read_fortran_field(const char* path, int nx, int ny, int nz, float* out) {
  std::ifstream in(path, std::ios::binary);
  if (!in) return false;
  int32_t n0, hdr[6], n1, m0, m1;
  in.read((char*)&n0, 4);
  in.read((char*)hdr, 24);
  in.read((char*)&n1, 4);
  if (n0 != 24 || n1 != 24 || hdr[0] != 1 || hdr[1] != nx || hdr[2] != 1 || hdr[3] != ny || hdr[4] != 1 ||
      hdr[5] != nz) {
    std::fprintf(stderr, "Wrong start file %s\n", path);
    return false;
  }
  in.read((char*)&m0, 4);
  in.read((char*)out, size_t(nx) * ny * nz * 4);
  in.read((char*)&m1, 4);
  return bool(in) && m0 == m1;
}

// Fortran unformatted sequential record pair of the *.init.bin files: a
// header record (1, nx, 1, ny, 1, nz) and the nx*ny*nz float32 block
bool write_fortran_field(const std::string& path, int nx, int ny, int nz, const float* a) {
  FILE* f = std::fopen(path.c_str(), "wb");
  if (!f) return false;
  const int32_t n0 = 24, hdr[6] = {1, nx, 1, ny, 1, nz};
  const int32_t m = int32_t(size_t(nx) * ny * nz * 4);
  bool ok = std::fwrite(&n0, 4, 1, f) == 1 && std::fwrite(hdr, 4, 6, f) == 6 && std::fwrite(&n0, 4, 1, f) == 1 &&
            std::fwrite(&m, 4, 1, f) == 1 && std::fwrite(a, 4, size_t(nx) * ny * nz, f) == size_t(nx) * ny * nz &&
            std::fwrite(&m, 4, 1, f) == 1;
  return std::fclose(f) == 0 && ok;
}

// write_fmtnumb (write_output.f90:858-875): six digits, zero-padded
std::string fmtnumb(int l) {
  char b[16];
  std::snprintf(b, sizeof b, "%06d", l);
  return b;
}

// read_and_setPops (main.CUF:2489-2529): q files popR.NNNNNN.init.bin and
// popB.NNNNNN.init.bin (direction l = 0 .. q-1) in directory dir, each one
// direction's nx*ny*nz populations; pR, pB get q planes of nx*ny*nz
bool read_init_pops(const std::string& dir, int q, int nx, int ny, int nz, std::vector<float>& pR,
                    std::vector<float>& pB) {
  const size_t n = size_t(nx) * ny * nz;
  pR.assign(size_t(q) * n, 0.f);
  pB.assign(size_t(q) * n, 0.f);
  for (int l = 0; l < q; ++l) {
    const std::string fr = dir + "/popR." + fmtnumb(l) + ".init.bin", fb = dir + "/popB." + fmtnumb(l) + ".init.bin";
    if (!read_fortran_field(fr.c_str(), nx, ny, nz, pR.data() + size_t(l) * n) ||
        !read_fortran_field(fb.c_str(), nx, ny, nz, pB.data() + size_t(l) * n)) {
      std::fprintf(stderr, "Wrong start pops file %s / %s\n", fr.c_str(), fb.c_str());
      return false;
    }
  }
  return true;
}

// the restart files of initType 4 (and 3): rhoR/rhoB.init.bin and the
// population files read_and_setPops reads, from the current state
bool write_restart(void* ctx, const std::string& dir, int q, int nx, int ny, int nz) {
  const size_t n = size_t(nx) * ny * nz;
  std::vector<float> pR(size_t(q) * n), pB(size_t(q) * n), R(n), B(n);
  if (lbx_get_pops(ctx, pR.data(), pB.data()) || lbx_get_fields(ctx, R.data(), B.data(), nullptr, nullptr))
    return false;
  bool ok = write_fortran_field(dir + "/rhoR.init.bin", nx, ny, nz, R.data()) &&
            write_fortran_field(dir + "/rhoB.init.bin", nx, ny, nz, B.data());
  for (int l = 0; ok && l < q; ++l)
    ok = write_fortran_field(dir + "/popR." + fmtnumb(l) + ".init.bin", nx, ny, nz, pR.data() + size_t(l) * n) &&
         write_fortran_field(dir + "/popB." + fmtnumb(l) + ".init.bin", nx, ny, nz, pB.data() + size_t(l) * n);
  return ok;
}

// initial densities of initType 1, 2, 3, 5, 6 (setupRho_Pops, main.CUF:2531-2608)
// densR / densB: the two-density model's droplet (setup2 with DIFFDENS,
// kernels_fluid_CG.CUF:163-169); 1, 1 otherwise
bool initial_fields(int type, int nx, int ny, int nz, unsigned seed, std::vector<float>& R, std::vector<float>& B,
                    float densR = 1.f, float densB = 1.f) {
  size_t n = size_t(nx) * ny * nz;
  R.assign(n, 0.f);
  B.assign(n, 0.f);
  // initType 3 starts from these densities; initType 4 reads them as well
  // (read_and_setRed_Blue) before its populations
  if (type == 3 || type == 4) {
    const bool ok = read_fortran_field("rhoR.init.bin", nx, ny, nz, R.data()) &&
                    read_fortran_field("rhoB.init.bin", nx, ny, nz, B.data());
    if (!ok) std::fprintf(stderr, "Wrong start rho file rhoR.init.bin / rhoB.init.bin\n");
    return ok;
  }
  std::mt19937_64 rng(seed);
  std::uniform_real_distribution<float> U(0.f, 1.f);
  for (int k = 1; k <= nz; ++k)
    for (int j = 1; j <= ny; ++j)
      for (int i = 1; i <= nx; ++i) {
        size_t h = size_t(i - 1) + size_t(nx) * (size_t(j - 1) + size_t(ny) * size_t(k - 1));
        float t;
        if (type == 1 || type == 5) {
          float radius = float(nz / 8);
          float dx = float(i) - float(nx / 2 + 0.5), dy = float(j) - float(ny / 2 + 0.5);
          float dz = (type == 1) ? float(k) - float(nz / 2 + 0.5) : 0.f;
          t = fcut(std::sqrt(dx * dx + dy * dy + dz * dz), radius, radius + 0.1f);
        } else if (type == 2) {
          t = (nz * 1 / 8 < k && k < nz * 5 / 8) ? 0.f : 1.f;
        } else if (type == 6) {
          t = 0.5f + 1.0e-4f * U(rng);
        } else {
          std::fprintf(stderr, "Wront init type= %d\n", type);
          return false;
        }
        R[h] = t;
        B[h] = 1.f - t;
        if (type == 1) {
          R[h] = t * densR;
          B[h] = (1.f - t) * densB;
        }
      }
  return true;
}

void write_vti(const std::string& fn, int nx, int ny, int nz, const std::vector<float>& R, const std::vector<float>& B,
               const std::vector<float>& V, const std::vector<float>& P) {
  FILE* f = std::fopen(fn.c_str(), "wb");
  if (!f) return;
  size_t n = size_t(nx) * ny * nz;
  uint64_t sz1 = n * 4, sz3 = 3 * n * 4;
  uint64_t off[4] = {0, 8 + sz1, 2 * (8 + sz1), 2 * (8 + sz1) + 8 + sz3};
  std::fprintf(f,
               "<?xml version=\"1.0\"?>\n<VTKFile type=\"ImageData\" version=\"1.0\" byte_order=\"LittleEndian\" "
               "header_type=\"UInt64\">\n<ImageData WholeExtent=\"1 %d 1 %d 1 %d\" Origin=\"0 0 0\" Spacing=\"1 1 1\">\n"
               "<Piece Extent=\"1 %d 1 %d 1 %d\">\n<PointData>\n",
               nx, ny, nz, nx, ny, nz);
  const char* names[4] = {"rhoR", "rhoB", "vel", "phase"};
  for (int a = 0; a < 4; ++a)
    std::fprintf(f, "<DataArray type=\"Float32\" Name=\"%s\" NumberOfComponents=\"%d\" format=\"appended\" offset=\"%llu\"/>\n",
                 names[a], a == 2 ? 3 : 1, (unsigned long long)off[a]);
  std::fprintf(f, "</PointData>\n</Piece>\n</ImageData>\n<AppendedData encoding=\"raw\">\n_");
  std::fwrite(&sz1, 8, 1, f); std::fwrite(R.data(), 4, n, f);
  std::fwrite(&sz1, 8, 1, f); std::fwrite(B.data(), 4, n, f);
  std::fwrite(&sz3, 8, 1, f); std::fwrite(V.data(), 4, 3 * n, f);
  std::fwrite(&sz1, 8, 1, f); std::fwrite(P.data(), 4, n, f);
  std::fprintf(f, "\n</AppendedData>\n</VTKFile>\n");
  std::fclose(f);
}

void write_particles_vtk(const std::string& fn, int n, const std::vector<double>& x, const std::vector<double>& v,
                         const std::vector<double>& q) {
  FILE* f = std::fopen(fn.c_str(), "w");
  if (!f) return;
  std::fprintf(f, "# vtk DataFile Version 2.0\nparticles\nASCII\nDATASET POLYDATA\nPOINTS %d float\n", n);
  for (int a = 0; a < n; ++a) std::fprintf(f, "%g %g %g\n", x[3 * a], x[3 * a + 1], x[3 * a + 2]);
  std::fprintf(f, "POINT_DATA %d\nVECTORS vel float\n", n);
  for (int a = 0; a < n; ++a) std::fprintf(f, "%g %g %g\n", v[3 * a], v[3 * a + 1], v[3 * a + 2]);
  std::fprintf(f, "VECTORS vx float\n");  // body x axis in the lab frame
  for (int a = 0; a < n; ++a) {
    const double* Q = &q[4 * a];
    std::fprintf(f, "%g %g %g\n", Q[0] * Q[0] + Q[1] * Q[1] - Q[2] * Q[2] - Q[3] * Q[3], 2 * (Q[1] * Q[2] + Q[0] * Q[3]),
                 2 * (Q[1] * Q[3] - Q[0] * Q[2]));
  }
  std::fclose(f);
}

int check(int rc, const char* what) {
  if (rc) std::fprintf(stderr, "%s: %s (%d)\n", what, lbx_error_string(rc), rc);
  return rc;
}

}  // namespace

int main(int argc, char** argv) {
  int nx = 64, ny = 64, nz = 64;
  const char* deck_path = "input.dat";
  const char* xyz_path = "input.xyz";
  std::string out = "output";
  unsigned seed = 1;
  std::string restart_out;
  lbx_params p;
  lbx_default_params(&p, nx, ny, nz);
  for (int a = 1; a < argc; ++a) {
    std::string s = argv[a];
    auto nxt = [&]() -> const char* { return a + 1 < argc ? argv[++a] : ""; };
    if (s == "-L") { nx = ny = nz = std::atoi(nxt()); }
    else if (s == "--nx") nx = std::atoi(nxt());
    else if (s == "--ny") ny = std::atoi(nxt());
    else if (s == "--nz") nz = std::atoi(nxt());
    else if (s == "--storage") {
      std::string t = nxt();
      p.storage = t == "f16" ? LBX_STORE_F16 : t == "bf16" ? LBX_STORE_BF16 : t == "f64" ? LBX_STORE_F64
                : t == "f16sd" ? LBX_STORE_F16_SD : t == "bf16sd" ? LBX_STORE_BF16_SD : LBX_STORE_F32;
    } else if (s == "--bgk") p.model = LBX_MODEL_BGK;
    else if (s == "--diffdens") {  // two fluid densities: --diffdens densR densB
      p.model = (p.model == LBX_MODEL_CG_D3Q27) ? LBX_MODEL_CG_DIFFDENS_D3Q27 : LBX_MODEL_CG_DIFFDENS;
      p.densR = float(std::atof(nxt()));
      p.densB = float(std::atof(nxt()));
    } else if (s == "--d3q27") {  // the D3Q27 lattice (with --diffdens: both)
      p.model = (p.model == LBX_MODEL_CG_DIFFDENS) ? LBX_MODEL_CG_DIFFDENS_D3Q27 : LBX_MODEL_CG_D3Q27;
    }
    else if (s == "--sigma") p.sigma = std::atof(nxt());
    else if (s == "--beta") p.beta = std::atof(nxt());
    else if (s == "--tau") p.tau = std::atof(nxt());
    else if (s == "--tauR") p.tauR = std::atof(nxt());
    else if (s == "--tauB") p.tauB = std::atof(nxt());
    else if (s == "--radius") p.radius = std::atof(nxt());
    else if (s == "--rmass") p.rmass = std::atof(nxt());
    else if (s == "--neutral") p.wetting = LBX_WET_NEUTRAL;
    else if (s == "--xyz") xyz_path = nxt();
    else if (s == "--out") out = nxt();
    else if (s == "--seed") seed = unsigned(std::atoi(nxt()));
    else if (s == "--restart-out") restart_out = nxt();
    else deck_path = argv[a];
  }
  p.nx = nx; p.ny = ny; p.nz = nz;
  Deck d;
  if (!read_deck(deck_path, d)) return 2;
  std::vector<double> x, v, q;
  if (d.withParticles) {
    if (!read_xyz(xyz_path, d.numAtoms, d.lrotate, x, v, q)) return 2;
    p.max_particles = d.numAtoms;
    p.lrotate = d.lrotate;
    p.max_vel = d.max_vel;
    for (int k = 0; k < 3; ++k) { p.ext_force[k] = d.ext_f[k]; p.ext_torque[k] = d.ext_t[k]; }
  }
  std::vector<float> R, B;
  if (!initial_fields(d.initType, nx, ny, nz, seed, R, B, p.densR, p.densB)) return 2;
  void* ctx = nullptr;
  if (check(lbx_create(&p, &ctx), "lbx_create")) return 1;
  if (check(lbx_set_fields(ctx, R.data(), B.data(), d.vx, d.vy, d.vz), "lbx_set_fields")) return 1;
  const int npop = (p.model == LBX_MODEL_CG_D3Q27 || p.model == LBX_MODEL_CG_DIFFDENS_D3Q27) ? 27 : 19;
  if (d.initType == 4) {
    std::vector<float> pR, pB;
    if (!read_init_pops(".", npop, nx, ny, nz, pR, pB)) return 2;
    if (check(lbx_set_pops(ctx, pR.data(), p.model == LBX_MODEL_BGK ? nullptr : pB.data()), "lbx_set_pops")) return 1;
  }
  if (d.withParticles && check(lbx_set_particles(ctx, d.numAtoms, x.data(), v.data(), nullptr, q.data()),
                               "lbx_set_particles"))
    return 1;
  mkdir(out.c_str(), 0755);
  size_t n = size_t(nx) * ny * nz;
  std::vector<float> V(3 * n), P(n);
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  double mlup_cells = double(n) / 1e6;
  double t_acc = 0;
  int since = 0;
  for (int step = 1; step <= d.nIter; ++step) {
    cudaEventRecord(e0, 0);
    double ms = 0;
    if (check(lbx_time_steps(ctx, 1, &ms, nullptr, nullptr), "lbx_step")) return 1;
    t_acc += ms;
    ++since;
    if (step % d.nIterOut == 0) {
      std::printf("Iter:%10d   Time(s):%10.4g   ms/it:%9.3g   Mlup/s:%8.0f\n", step, t_acc * 1e-3, t_acc / since,
                  mlup_cells * since / (t_acc * 1e-3));
      t_acc = 0;
      since = 0;
    }
    if (step % d.nIterVTK == 0) {
      if (check(lbx_get_fields(ctx, R.data(), B.data(), V.data(), P.data()), "lbx_get_fields")) return 1;
      char fn[512];
      std::snprintf(fn, sizeof fn, "%s/rho_0.%08d.vti", out.c_str(), step);
      write_vti(fn, nx, ny, nz, R, B, V, P);
      if (d.withParticles) {
        if (check(lbx_get_particles(ctx, x.data(), v.data(), nullptr, q.data(), nullptr, nullptr),
                  "lbx_get_particles"))
          return 1;
        std::snprintf(fn, sizeof fn, "%s/particle_0.%08d.vtk", out.c_str(), step);
        write_particles_vtk(fn, d.numAtoms, x, v, q);
      }
    }
  }
  if (!restart_out.empty()) {
    mkdir(restart_out.c_str(), 0755);
    if (!write_restart(ctx, restart_out, npop, nx, ny, nz)) {
      std::fprintf(stderr, "restart files not written to %s\n", restart_out.c_str());
      lbx_destroy(ctx);
      return 1;
    }
  }
  int32_t code = 0, st = 0;
  int64_t where = 0;
  lbx_status(ctx, &code, &st, &where);
  lbx_destroy(ctx);
  if (code) {
    std::fprintf(stderr, "device error %d (%s) at step %d, index %lld\n", code, lbx_error_string(code), st,
                 (long long)where);
    return 3;
  }
  return 0;
}
