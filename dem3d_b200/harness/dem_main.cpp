// The time loop of DEM3D's main program (src/DEM.f90:85-99) in C++ over the
// C-ABI: MethodOrder-1 Euler start-up steps, then for every step a pouring
// attempt every IPouring steps (PouringAttempt), MoveParticles and
// UpdateParticleList.  The spec parser, periodic tasks and reports stay with
// the reference.
//
//   dem_main <case.bin> <out.bin>
//
// case.bin: the dem_params struct as laid out by dem3d_b200.h, then int32 n,
// int32 number_of_steps, int32 pouring_interval (0: none), int32 has_radius,
// comp[n] (int32), radius[n] if has_radius, pos[3n], vel[3n], omega[3n]
// (rows of three doubles); with pouring, a dem_pouring struct follows.
// out.bin: int32 n, pos[3n], vel[3n], omega[3n], comp[n] (int32), int64 Ncol.
// Exit status: 0 done, 1 failure, 2 bad arguments or files, 3 no CUDA device.
#include <cstdio>
#include <vector>

#include "../../include/dem3d_b200.hpp"

namespace {

bool read_all(std::FILE* f, void* dst, size_t bytes) { return std::fread(dst, 1, bytes, f) == bytes; }

}  // namespace

int main(int argc, char** argv) {
  if (argc != 3) {
    std::fprintf(stderr, "usage: %s <case.bin> <out.bin>\n", argv[0]);
    return 2;
  }
  std::FILE* in = std::fopen(argv[1], "rb");
  if (!in) {
    std::fprintf(stderr, "cannot open %s\n", argv[1]);
    return 2;
  }
  dem_params p{};
  int32_t head[4] = {0, 0, 0, 0};  // n, number_of_steps, pouring_interval, has_radius
  bool ok = read_all(in, &p, sizeof(p)) && read_all(in, head, sizeof(head));
  const int n = head[0], steps = head[1], pour_every = head[2], has_radius = head[3];
  ok = ok && n >= 0 && steps >= 0 && pour_every >= 0;
  std::vector<int32_t> comp(ok ? (size_t)n : 0);
  std::vector<double> radius(ok && has_radius ? (size_t)n : 0);
  std::vector<double> pos(ok ? 3 * (size_t)n : 0), vel(pos.size()), omega(pos.size());
  dem_pouring pouring{};
  ok = ok && read_all(in, comp.data(), comp.size() * sizeof(int32_t)) &&
       read_all(in, radius.data(), radius.size() * sizeof(double)) &&
       read_all(in, pos.data(), pos.size() * sizeof(double)) &&
       read_all(in, vel.data(), vel.size() * sizeof(double)) &&
       read_all(in, omega.data(), omega.size() * sizeof(double)) &&
       (pour_every == 0 || read_all(in, &pouring, sizeof(pouring)));
  std::fclose(in);
  if (!ok) {
    std::fprintf(stderr, "%s: not a case file\n", argv[1]);
    return 2;
  }
  try {
    dem3d::System s(p);
    s.SetState(n, has_radius ? nullptr : comp.data(), has_radius ? radius.data() : nullptr,
               pos.data(), vel.data(), omega.data());
    s.InitializeCellDistribution();
    if (pour_every > 0) s.SetPouring(pouring);
    // MethodOrder-1 Euler steps whatever NumberOfSteps is (src/DEM.f90:88-90)
    for (int step = 1; step <= p.method_order - 1; step++) s.MoveParticlesEuler();
    for (int step = p.method_order; step <= steps; step++) {
      if (pour_every > 0 && step % pour_every == 0) s.PourParticle();
      s.MoveParticles(step);
      s.UpdateParticleList();
    }
    dem3d::Particles out;
    s.GetParticles(out);
    const std::vector<int32_t> c = s.Components();
    const int32_t m = (int32_t)c.size();
    const int64_t ncol = s.Ncol();
    std::FILE* f = std::fopen(argv[2], "wb");
    if (!f) {
      std::fprintf(stderr, "cannot write %s\n", argv[2]);
      return 2;
    }
    std::fwrite(&m, sizeof(m), 1, f);
    std::fwrite(out.pos.data(), sizeof(double), out.pos.size(), f);
    std::fwrite(out.vel.data(), sizeof(double), out.vel.size(), f);
    std::fwrite(out.omega.data(), sizeof(double), out.omega.size(), f);
    std::fwrite(c.data(), sizeof(int32_t), c.size(), f);
    std::fwrite(&ncol, sizeof(ncol), 1, f);
    std::fclose(f);
    std::printf("steps %d particles %d Ncol %lld\n", steps, m, (long long)ncol);
  } catch (const dem3d::Error& e) {
    std::fprintf(stderr, "%s\n", e.what());
    return e.code == DEM_ERR_NO_DEVICE ? 3 : 1;
  }
  return 0;
}
