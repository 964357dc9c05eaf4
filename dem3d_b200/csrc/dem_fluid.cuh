// Fluid drag (mFluid, src/mFluid.f90) on the device.  Before a pass on a
// side, k_fluid_levels averages the spheres' cross-sections and upward
// velocities over the NL+1 horizontal levels (UpdateVelocityField, :96-139)
// and k_fluid_drag evaluates DragForce (:143-197) for every sphere; the pass
// kernel adds it to the sphere's own force where ComputeAccelerations does
// (src/MForces.f90:316).  The level sums use a fixed summation tree, so the
// result is deterministic; it differs from the reference's index-ordered
// sums and from its libm pow in the last bits only.
#pragma once

#include "dem_kernels.cuh"

namespace dem {

constexpr int FLUID_THREADS = 256;

struct FluidArgs {
  int levels;     // NL
  double dz;      // Delta_Z = Lbox(3)/NL
  double h2;      // H_2 = Lbox(3)/2
  double vf0;     // Vf0 = FluidFlowRate/Area
  double area;    // Lbox(1)*Lbox(2)
  double density;
  double viscosity;
  double comp_density[NCM];
  double comp_radius[NCM];
};

// one block per level: per-thread sums over a fixed particle subset, then a
// fixed tree over the block
__global__ void __launch_bounds__(FLUID_THREADS) k_fluid_levels(
    FluidArgs F, int n, const double* __restrict__ pz, const double* __restrict__ vz,
    const int* __restrict__ comp, double* __restrict__ vf, double* __restrict__ ef,
    const Counters* __restrict__ cnt) {
  if (cnt->abort) return;
  __shared__ double sa[FLUID_THREADS], sb[FLUID_THREADS], sc[FLUID_THREADS];
  const int k = blockIdx.x;
  const double Pi = 3.1415926535897932384626433832795;
  const double Zk = -F.h2 + (double)k * F.dz;
  double A = 0.0, B = 0.0, C = 0.0;
  for (int i = threadIdx.x; i < n; i += FLUID_THREADS) {
    const int ind = comp[i];
    const double d = Zk - pz[i];
    const double Diff2 = d * d;
    const double R = F.comp_radius[ind];
    const double R2 = R * R;
    if (Diff2 < R2) {
      const double Ai = Pi * (R2 - Diff2);
      A = A + Ai;
      const double DensAi = Ai * F.comp_density[ind];
      B = B + DensAi * vz[i];
      C = C + DensAi;
    }
  }
  sa[threadIdx.x] = A;
  sb[threadIdx.x] = B;
  sc[threadIdx.x] = C;
  __syncthreads();
  for (int s = FLUID_THREADS / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) {
      sa[threadIdx.x] += sa[threadIdx.x + s];
      sb[threadIdx.x] += sb[threadIdx.x + s];
      sc[threadIdx.x] += sc[threadIdx.x + s];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    const double SumA = sa[0], SumB = sb[0], SumC = sc[0];
    if (SumA == 0.0) {
      vf[k] = F.vf0;
      ef[k] = 1.0;
    } else {
      const double Es = SumA / F.area;
      const double Ef = 1.0 - Es;
      ef[k] = Ef;
      const double Vs = SumB / SumC;
      vf[k] = (F.vf0 - Es * Vs) / Ef;
    }
  }
}

// DragForce for every sphere (the level index kept inside 0..NL-1, where the
// reference would read past Vf(NL) for a sphere above the box)
__global__ void k_fluid_drag(FluidArgs F, int n, StateArrays Q, const int* __restrict__ comp,
                             const double* __restrict__ vf, const double* __restrict__ ef,
                             double* __restrict__ drag, const Counters* __restrict__ cnt) {
  if (cnt->abort) return;
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  const double Zi = Q.pz[p];
  const double jr = (Zi + F.h2) / F.dz;
  int j = (int)jr;
  j = j < 0 ? 0 : (j > F.levels - 1 ? F.levels - 1 : j);
  double Vfz = vf[j];
  Vfz = Vfz + (jr - (double)j) * (vf[j + 1] - Vfz);
  double Efz = ef[j];
  Efz = Efz + (jr - (double)j) * (ef[j + 1] - Efz);
  double Vr[3] = {-Q.vx[p], -Q.vy[p], -Q.vz[p]};
  Vr[2] = Vfz + Vr[2];
  const double Vra = sqrt((Vr[0] * Vr[0] + Vr[1] * Vr[1]) + Vr[2] * Vr[2]);
  double FD[3] = {0.0, 0.0, 0.0};
  if (Vra > 0.0) {
    const double Ri = F.comp_radius[comp[p]];
    const double Re = 2.0 * Efz * Ri * Vra * F.density / F.viscosity;
    double nn = 3.6, n0 = nn + 1.0, x = 0.0;
    for (int it = 0; fabs(nn - n0) > 1.e-8 && it < 1000; it++) {
      n0 = nn;
      x = Re / pow(Efz, nn);
      const double x75 = pow(x, 0.75);
      nn = (4.8 + 0.42 * x75) / (1.0 + 0.175 * x75);
    }
    double a = 0.63 + 4.8 / sqrt(x);
    const double Cd1 = a * a;
    a = 0.63 + 4.8 / sqrt(Re);
    const double CD = a * a;
    const double fi = (Cd1 / CD) * pow(Efz, 2.0 * (1.0 - nn));
    const double Pi = 3.1415926535897932384626433832795;
    const double s = CD * (Pi / 2.0) * Ri * Ri * F.density * Vra;
#pragma unroll
    for (int k = 0; k < 3; k++) FD[k] = s * Vr[k] * fi;
  }
#pragma unroll
  for (int k = 0; k < 3; k++) drag[(size_t)3 * p + k] = FD[k];
}

}  // namespace dem
