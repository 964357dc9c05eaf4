// dem3d_b200.hpp -- C++ host side over the C-ABI of dem3d_b200.h.
//
// dem3d::System mirrors the module routines of DEM3D's per-step path with
// their names and argument meaning (InitializeCellDistribution,
// ComputeAccelerations, MoveParticlesEuler, MoveParticles,
// UpdateParticleList, PourParticle).  Where the reference stops the program
// on an error, a failing call throws dem3d::Error with the library's status
// code and message.  Header only; link against libdem3d_b200.so.
#ifndef DEM3D_B200_HPP
#define DEM3D_B200_HPP

#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

#include "dem3d_b200.h"

namespace dem3d {

class Error : public std::runtime_error {
 public:
  Error(int status, const std::string& what) : std::runtime_error(what), code(status) {}
  int code;  // DEM_ERR_*
};

// Particle(1:NP) (TParticle, src/MDimension3D.f90:28-35) as rows of three.
struct Particles {
  std::vector<double> pos, vel, omega, acc, alpha;
  void resize(int n) {
    for (std::vector<double>* v : {&pos, &vel, &omega, &acc, &alpha}) v->assign(3 * (size_t)n, 0.0);
  }
};

class System {
 public:
  // InitializeAuxiliaries (src/MDEM.f90:110-162) for the scaled parameters.
  explicit System(const dem_params& params) {
    const int st = dem_create(&params, &ctx_);
    if (st != DEM_OK)
      throw Error(st, st == DEM_ERR_NO_DEVICE ? "dem_create: no CUDA device"
                                              : "dem_create failed: " + std::to_string(st));
  }
  ~System() {
    if (ctx_) dem_destroy(ctx_);  // FinalizeDEM
  }
  System(const System&) = delete;
  System& operator=(const System&) = delete;

  // Particle(1:NP) with InitializeIntegrationVariables and InitializeContacts.
  // comp: component per particle (NULL in per-particle-radius mode); radius:
  // per-particle radius (NULL in component mode).
  void SetState(int n, const int32_t* comp, const double* radius, const double* pos,
                const double* vel, const double* omega) {
    check(dem_set_state(ctx_, n, comp, radius, pos, vel, omega, nullptr, nullptr), "SetState");
  }
  void InitializeCellDistribution() {
    check(dem_initialize_cell_distribution(ctx_), "InitializeCellDistribution");
  }
  void ComputeAccelerations(bool predicted, double time_step, bool update) {
    check(dem_compute_accelerations(ctx_, predicted ? 1 : 0, time_step, update ? 1 : 0),
          "ComputeAccelerations");
  }
  // The same pass, also returning its Force and Torque arrays (rows of three,
  // before the division by mass and inertia).
  void ComputeForces(bool predicted, double time_step, bool update, std::vector<double>& force,
                     std::vector<double>& torque) {
    force.assign(3 * (size_t)NP(), 0.0);
    torque.assign(force.size(), 0.0);
    check(dem_compute_forces(ctx_, predicted ? 1 : 0, time_step, update ? 1 : 0, force.data(),
                             torque.data()),
          "ComputeForces");
  }
  void MoveParticlesEuler() { check(dem_move_particles_euler(ctx_), "MoveParticlesEuler"); }
  void MoveParticles(int step) { check(dem_move_particles(ctx_, step), "MoveParticles"); }
  // Returns the number of particles removed.
  int64_t UpdateParticleList() {
    int64_t removed = 0;
    check(dem_update_particle_list(ctx_, &removed), "UpdateParticleList");
    return removed;
  }
  // Returns whether a particle was inserted.
  bool PourParticle() {
    int32_t inserted = 0;
    check(dem_pour_particle(ctx_, &inserted), "PourParticle");
    return inserted != 0;
  }
  void SetPouring(const dem_pouring& pouring) { check(dem_set_pouring(ctx_, &pouring), "SetPouring"); }
  void SetWallMotion(const dem_wall_motion* motion) {
    check(dem_set_wall_motion(ctx_, motion), "SetWallMotion");
  }
  int NP() {
    int32_t n = 0;
    check(dem_get_n(ctx_, &n), "NP");
    return n;
  }
  void GetParticles(Particles& out) {
    out.resize(NP());
    check(dem_get_state(ctx_, out.pos.data(), out.vel.data(), out.omega.data(), out.acc.data(),
                        out.alpha.data()),
          "GetParticles");
  }
  // Component index of every particle (Particle%Index - 1), after removals
  // and insertions.
  std::vector<int32_t> Components() {
    std::vector<int32_t> comp((size_t)NP());
    check(dem_get_components(ctx_, comp.data()), "Components");
    return comp;
  }
  int64_t Ncol() {
    int64_t ncol = 0;
    check(dem_get_ncol(ctx_, &ncol), "Ncol");
    return ncol;
  }
  dem_observables Observables() {
    dem_observables o{};
    check(dem_get_observables(ctx_, &o), "Observables");
    return o;
  }
  dem_ctx* handle() { return ctx_; }

 private:
  void check(int status, const char* routine) {
    if (status != DEM_OK) throw Error(status, std::string(routine) + ": " + dem_last_error(ctx_));
  }
  dem_ctx* ctx_ = nullptr;
};

}  // namespace dem3d

#endif
