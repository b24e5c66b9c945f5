// SCF potential build and Pulay mixing on the device: the per-iteration work around the eigensolver
// and density path (scf/scf.zig:148-188), kept next to the data so the density, the potential and
// the mixing history never leave HBM between iterations.
//
//   dftcuda_hxc_potential   build_potential_grid (scf/potential.zig:144-203): FFT of rho, Hartree
//                           8 pi rho(G)/G^2 (hartree_potential_at_g, potential.zig:34-44), LDA-PZ
//                           (xc/xc.zig:195-211, 344-384) or PBE (xc.zig:213-342 with the gradient
//                           assembly of scf/xc_fields.zig:108-142, 306-375) f and V_xc and the FFT
//                           of V_xc; energy terms of scf/energy.zig:372-396 from the same passes
//   dftcuda_potential_real  V(r) = V_loc(r) + FFT^-1 V(G) (build_local_potential_real,
//                           potential.zig:320-334)
//   dftcuda_ionic_potential V_ion(G) and V_loc(r) (build_ionic_potential_grid, potential.zig:279-318)
//                           with the analytic GTH local form factor
//   dftcuda_pulay_mix       PulayMixer.mix_with_residual (scf/mixing.zig:182-248) with the bordered
//                           system solved as solve_pulay_system (mixing.zig:341-405)
//
// Bounds: every kernel here streams N-point fields once or twice (HBM bound); the FFTs are the
// library's axis passes.  Sums are taken as fixed per-block partials added on the host in block
// order, so results do not depend on scheduling.
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include "kctx.cuh"

namespace dftcuda {
namespace {

constexpr int kPotThreads = 256;
constexpr int kPotBlocks = 592;  // 4 per SM on 148 SMs; per-block partial sums
constexpr double kPi = 3.14159265358979323846;

__global__ void k_pot_g2(int nx, int ny, int nz, double b00, double b01, double b02, double b10, double b11, double b12,
                         double b20, double b21, double b22, double* __restrict__ g2) {
  const long N = (long)nx * ny * nz;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < N; i += (long)gridDim.x * blockDim.x) {
    const int x = (int)(i % nx), y = (int)((i / nx) % ny), z = (int)(i / ((long)nx * ny));
    const double h = x < (nx + 1) / 2 ? x : x - nx;
    const double k = y < (ny + 1) / 2 ? y : y - ny;
    const double l = z < (nz + 1) / 2 ? z : z - nz;
    const double gx = h * b00 + k * b10 + l * b20;
    const double gy = h * b01 + k * b11 + l * b21;
    const double gz = h * b02 + k * b12 + l * b22;
    g2[i] = gx * gx + gy * gy + gz * gz;
  }
}

// LDA-PZ in Ry: f (energy per volume) and v = df/dn; zero for n <= 1e-12 (xc.zig:195-211, 344-384).
__device__ __forceinline__ void lda_pz(double n, double& f, double& v) {
  if (n <= 1e-12) {
    f = 0.0;
    v = 0.0;
    return;
  }
  const double n13 = pow(n, 1.0 / 3.0);
  const double c_x = -0.75 * pow(3.0 / kPi, 1.0 / 3.0);
  const double ex = n * c_x * n13;
  const double rs = pow(3.0 / (4.0 * kPi * n), 1.0 / 3.0);
  double eps_c, v_c;
  if (rs < 1.0) {
    const double a = 0.0311, b = -0.048, c = 0.0020, d = -0.0116;
    const double lr = log(rs);
    eps_c = a * lr + b + c * rs * lr + d * rs;
    const double de = a / rs + c * lr + c + d;
    v_c = eps_c - (rs / 3.0) * de;
  } else {
    const double g = -0.1423, b1 = 1.0529, b2 = 0.3334;
    const double sr = sqrt(rs);
    const double den = 1.0 + b1 * sr + b2 * rs;
    eps_c = g / den;
    const double de = -g * (0.5 * b1 / sr + b2) / (den * den);
    v_c = eps_c - (rs / 3.0) * de;
  }
  f = 2.0 * (ex + n * eps_c);
  v = 2.0 * (4.0 / 3.0 * c_x * n13 + v_c);
}

__device__ __forceinline__ double block_sum(double v, double* red) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) red[w] = v;
  __syncthreads();
  double t = 0.0;
  if (threadIdx.x == 0)
    for (int i = 0; i < kPotThreads / 32; ++i) t += red[i];
  return t;
}

// a = rho (complex), b = V_xc (complex); part[block] = sum of f_xc over the block's points.
__global__ void __launch_bounds__(kPotThreads) k_pot_xc(const double* __restrict__ rho, long N, double2* __restrict__ a,
                                                        double2* __restrict__ b, double* __restrict__ part) {
  __shared__ double red[kPotThreads / 32];
  double s = 0.0;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < N; i += (long)gridDim.x * blockDim.x) {
    const double n = rho[i];
    double f, v;
    lda_pz(n, f, v);
    a[i] = make_double2(n, 0.0);
    b[i] = make_double2(v, 0.0);
    s += f;
  }
  s = block_sum(s, red);
  if (threadIdx.x == 0) part[blockIdx.x] = s;
}

// a = N rho(G), b = N V_xc(G) (unnormalised forward FFTs).  out = V_H + V_xc (normalised);
// part[0][block] = sum 8 pi |rho(G)|^2 / G^2, part[1][block] = sum Re(v_in(G) conj(rho(G))).
__global__ void __launch_bounds__(kPotThreads) k_pot_hartree(const double2* __restrict__ a, const double2* __restrict__ b,
                                                             const double* __restrict__ g2, long N,
                                                             const double2* __restrict__ v_in, double2* __restrict__ out,
                                                             double* __restrict__ part) {
  __shared__ double red[kPotThreads / 32];
  const double inv = 1.0 / (double)N;
  double eh = 0.0, ei = 0.0;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < N; i += (long)gridDim.x * blockDim.x) {
    const double2 rg = make_double2(a[i].x * inv, a[i].y * inv);
    const double q = g2[i];
    double2 v = make_double2(b[i].x * inv, b[i].y * inv);
    if (q > 1e-12) {
      const double k = 8.0 * kPi / q;
      v.x += k * rg.x;
      v.y += k * rg.y;
      eh += k * (rg.x * rg.x + rg.y * rg.y);
    }
    out[i] = v;
    if (v_in) {
      const double2 w = v_in[i];
      ei += w.x * rg.x + w.y * rg.y;
    }
  }
  eh = block_sum(eh, red);
  ei = block_sum(ei, red);
  if (threadIdx.x == 0) {
    part[blockIdx.x] = eh;
    part[kPotBlocks + blockIdx.x] = ei;
  }
}

// Ionic local potential in G space (build_ionic_potential_grid, scf/potential.zig:279-318):
// V(G) = (2 / Omega) sum_atoms ff_s(|G|) e^{-i G . tau} for 1e-12 < G^2 <= g2max, else 0, with the
// analytic local form factor of Goedecker-Teter-Hutter pseudopotentials (Hartree, hence the 2 for Ry):
//   ff(G) = -4 pi Z / G^2 e^{-x} + sqrt(8 pi^3) r^3 e^{-x} [C1 + C2 (3 - y) + C3 (15 - 10 y + y^2)
//           + C4 (105 - 105 y + 21 y^2 - y^3)],  y = G^2 r^2, x = y / 2.
// One thread per G point; atom positions and species parameters in shared memory.
constexpr int kIonMaxSpecies = 8;
constexpr int kIonAtomTile = 512;

// Local form factor of a species in Ry, either the analytic GTH form above (gth != nullptr, 6
// parameters per species) or values precomputed per box point (vq[s * N + i], from the species'
// radial mesh by k_pot_vq_radial).  keep() is the G-vector selection of each: GTH
// 1e-12 < G^2 <= g2max; radial |G| >= 1e-10 and G^2 < g2max (build_ionic_potential_grid,
// potential.zig:291-306, and ionic_local_potential_with_table, hamiltonian.zig).
struct LocalFF {
  const double* gth = nullptr;
  const double* vq = nullptr;
  long N = 0;
  __device__ bool keep(double g2, double g2max) const {
    return vq ? (sqrt(g2) >= 1e-10 && g2 < g2max) : (g2 > 1e-12 && g2 <= g2max);
  }
  __device__ double ry(int s, double g2, long i) const {
    if (vq) return vq[(long)s * N + i];
    const double Z = gth[6 * s], r = gth[6 * s + 1];
    const double c1 = gth[6 * s + 2], c2 = gth[6 * s + 3], c3 = gth[6 * s + 4], c4 = gth[6 * s + 5];
    const double yy = g2 * r * r, e = exp(-0.5 * yy);
    const double poly = c1 + c2 * (3.0 - yy) + c3 * (15.0 - 10.0 * yy + yy * yy) +
                        c4 * (105.0 - 105.0 * yy + 21.0 * yy * yy - yy * yy * yy);
    return 2.0 * (-4.0 * kPi * Z / g2 * e + sqrt(8.0 * kPi * kPi * kPi) * r * r * r * e * poly);
  }
};

// local_vq_short_range (form_factor.zig:223-262, the default local_potential mode of
// config/defaults.zig:28) at every box point, per species:
//   vq[s][i] = 4 pi sum_j r_j^2 [V_loc(r_j) + 2 Z / r_j] sinc(|G_i| r_j) rab_j w_j - 8 pi Z / |G_i|^2  (Ry)
// summed in mesh order like the reference's loop, the 2Z/r term skipped at r < 1e-10 and the
// Coulomb term at |G| < 1e-10; w the composite-trapezoid weights of radial_integration.zig:7-13.
// Species s uses mesh points [off[s], off[s+1]); every thread of a warp reads the same mesh entry.
__global__ void __launch_bounds__(kPotThreads) k_pot_vq_radial(const double* __restrict__ g2, long N, int nspecies,
                                                               const int* __restrict__ off, const double* __restrict__ r,
                                                               const double* __restrict__ rab, const double* __restrict__ vloc,
                                                               const double* __restrict__ zval, double* __restrict__ vq) {
  const double cw[5] = {23.75 / 72.0, 95.10 / 72.0, 55.20 / 72.0, 79.30 / 72.0, 70.65 / 72.0};
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < N; i += (long)gridDim.x * blockDim.x) {
    const double q = sqrt(g2[i]);
    for (int s = 0; s < nspecies; ++s) {
      const int j0 = off[s], n = off[s + 1] - j0;
      const double z = zval[s];
      double sum = 0.0;
      for (int jj = 0; jj < n; ++jj) {
        double w = 1.0;
        if (n >= 10) {
          if (jj < 5) w = cw[jj];
          else if (jj >= n - 5) w = cw[n - 1 - jj];
        }
        const double rj = __ldg(r + j0 + jj);
        const double vc = rj < 1e-10 ? 0.0 : 2.0 * z / rj;
        const double x = q * rj;
        const double sinc = fabs(x) < 1e-12 ? 1.0 : sin(x) / x;
        sum += rj * rj * (__ldg(vloc + j0 + jj) + vc) * sinc * __ldg(rab + j0 + jj) * w;
      }
      double v = 4.0 * kPi * sum;
      if (q >= 1e-10) v -= 8.0 * kPi * z / (q * q);
      vq[(long)s * N + i] = v;
    }
  }
}
__global__ void __launch_bounds__(kPotThreads) k_pot_ionic(const double* __restrict__ g2, int nx, int ny, int nz, double b00,
                                                           double b01, double b02, double b10, double b11, double b12,
                                                           double b20, double b21, double b22, int nspecies,
                                                           LocalFF ff, int natoms,
                                                           const int* __restrict__ species, const double* __restrict__ pos,
                                                           double g2max, double inv_volume, double2* __restrict__ out) {
  __shared__ double sx[kIonAtomTile], sy[kIonAtomTile], sz[kIonAtomTile];
  __shared__ int ss[kIonAtomTile];
  const long N = (long)nx * ny * nz;
  const long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
  double gx = 0.0, gy = 0.0, gz = 0.0, q = 0.0;
  if (i < N) {
    const int x = (int)(i % nx), y = (int)((i / nx) % ny), z = (int)(i / ((long)nx * ny));
    const double h = x < (nx + 1) / 2 ? x : x - nx;
    const double k = y < (ny + 1) / 2 ? y : y - ny;
    const double l = z < (nz + 1) / 2 ? z : z - nz;
    gx = h * b00 + k * b10 + l * b20;
    gy = h * b01 + k * b11 + l * b21;
    gz = h * b02 + k * b12 + l * b22;
    q = g2[i];
  }
  double sre[kIonMaxSpecies], sim[kIonMaxSpecies];
#pragma unroll
  for (int s = 0; s < kIonMaxSpecies; ++s) sre[s] = sim[s] = 0.0;
  for (int a0 = 0; a0 < natoms; a0 += kIonAtomTile) {
    const int na = min(kIonAtomTile, natoms - a0);
    __syncthreads();
    for (int t = threadIdx.x; t < na; t += blockDim.x) {
      sx[t] = pos[3 * (a0 + t)];
      sy[t] = pos[3 * (a0 + t) + 1];
      sz[t] = pos[3 * (a0 + t) + 2];
      ss[t] = species[a0 + t];
    }
    __syncthreads();
    for (int t = 0; t < na; ++t) {
      double sn, cs;
      sincos(gx * sx[t] + gy * sy[t] + gz * sz[t], &sn, &cs);
      const int sp = ss[t];
#pragma unroll
      for (int s = 0; s < kIonMaxSpecies; ++s)
        if (s == sp) {
          sre[s] += cs;
          sim[s] -= sn;  // e^{-i G . tau}
        }
    }
  }
  if (i >= N) return;
  double2 v = make_double2(0.0, 0.0);
  if (ff.keep(q, g2max)) {
    for (int s = 0; s < nspecies; ++s) {
      const double w = ff.ry(s, q, i) * inv_volume;
      v.x += w * sre[s];
      v.y += w * sim[s];
    }
  }
  out[i] = v;
}

// ---- PBE (generalised-gradient) exchange-correlation -------------------------------------------
// Point functional of xc/xc.zig:213-342 (pbe, pbe_exchange, pbe_correlation, pw92_correlation), in
// Ry: f per volume, df/dn and df/dg2 with g2 = |grad n|^2; all zero for n <= 1e-12.
__device__ void pbe_point(double n, double g2, double& f, double& vn, double& vg) {
  if (n <= 1e-12) {
    f = vn = vg = 0.0;
    return;
  }
  // exchange
  const double mu = 0.2195149727645171, kappa = 0.804;
  const double c_x = -0.75 * pow(3.0 / kPi, 1.0 / 3.0);
  const double n13 = pow(n, 1.0 / 3.0);
  const double ex0 = n * c_x * n13;
  const double kf = pow(3.0 * kPi * kPi * n, 1.0 / 3.0);
  const double den_x = 4.0 * kf * kf * n * n;
  const double s2 = (g2 > 0.0 && den_x > 0.0) ? g2 / den_x : 0.0;
  const double t = 1.0 + mu * s2 / kappa;
  const double fx = 1.0 + kappa - kappa / t;
  const double dfs = mu / (t * t);
  const double ex_dn = 4.0 / 3.0 * c_x * n13 * fx + ex0 * dfs * (-8.0 / 3.0 * s2 / n);
  const double ex_dg = ex0 * dfs * (den_x > 0.0 ? 1.0 / den_x : 0.0);
  // correlation: PW92 local part and the PBE gradient term H
  const double beta = 0.06672455060314922, gamma = 0.031090690869654895;
  const double rs = pow(3.0 / (4.0 * kPi * n), 1.0 / 3.0);
  double eps_c = 0.0, deps_drs = 0.0;
  if (rs > 1e-12) {
    const double a = 0.031091, a1 = 0.21370, b1 = 7.5957, b2 = 3.5876, b3 = 1.6382, b4 = 0.49294;
    const double sq = sqrt(rs);
    const double ff = b1 * sq + b2 * rs + b3 * rs * sq + b4 * rs * rs;
    const double gg = 1.0 + 1.0 / (2.0 * a * ff);
    const double lg = log(gg);
    eps_c = -2.0 * a * (1.0 + a1 * rs) * lg;
    const double dfr = 0.5 * b1 / sq + b2 + 1.5 * b3 * sq + 2.0 * b4 * rs;
    const double dlg = -(1.0 / (2.0 * a * ff * ff * gg)) * dfr;
    deps_drs = -2.0 * a * (a1 * lg + (1.0 + a1 * rs) * dlg);
  }
  const double v_c = eps_c - (rs / 3.0) * deps_drs;
  const double deps_dn = deps_drs * (-rs / (3.0 * n));
  const double ks2 = 4.0 * kf / kPi;
  const double den_c = 4.0 * ks2 * n * n;
  const double t2 = (g2 > 0.0 && den_c > 0.0) ? g2 / den_c : 0.0;
  const double bg = beta / gamma;
  const double x = bg * t2;
  const double u = exp(-eps_c / gamma);
  const double um = u - 1.0;
  const bool big = fabs(um) > 1e-12;
  const double A = big ? bg / um : 0.0;
  const double y = A * t2;
  const double d2 = 1.0 + y + y * y;
  const double q = (1.0 + y) / d2;
  const double arg = 1.0 + x * q;
  const double H = arg > 0.0 ? gamma * log(arg) : 0.0;
  const double d2s = d2 * d2;
  const double dq_dt2 = -A * y * (2.0 + y) / d2s;
  const double darg = bg * q + x * dq_dt2;
  const double dH_dt2 = arg > 0.0 ? gamma * darg / arg : 0.0;
  const double dH_dA = arg > 0.0 ? -gamma * x * t2 * y * (2.0 + y) / (arg * d2s) : 0.0;
  const double dA_dn = big ? bg * u / (gamma * um * um) * deps_dn : 0.0;
  const double dH_dn = dH_dt2 * (-7.0 / 3.0 * t2 / n) + dH_dA * dA_dn;
  const double dH_dg = dH_dt2 * (den_c > 0.0 ? 1.0 / den_c : 0.0);
  f = 2.0 * (ex0 * fx + n * (eps_c + H));
  vn = 2.0 * (ex_dn + v_c + H + n * dH_dn);
  vg = 2.0 * (ex_dg + n * dH_dg);
}

struct Recip9 {
  double b[9];  // rows b1, b2, b3
};

// Cartesian component d of the G vector of box point i (FFT order, x fastest).
__device__ __forceinline__ double pot_gcomp(long i, int nx, int ny, int nz, const Recip9& r, int d) {
  const int x = (int)(i % nx), y = (int)((i / nx) % ny), z = (int)(i / ((long)nx * ny));
  const double h = x < (nx + 1) / 2 ? x : x - nx;
  const double k = y < (ny + 1) / 2 ? y : y - ny;
  const double l = z < (nz + 1) / 2 ? z : z - nz;
  return h * r.b[d] + k * r.b[3 + d] + l * r.b[6 + d];
}

__global__ void k_pot_to_complex(const double* __restrict__ x, long N, double2* __restrict__ out) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < N; i += (long)gridDim.x * blockDim.x)
    out[i] = make_double2(x[i], 0.0);
}

// out (=, or += when accumulate) i G_d in (gradient_from_real / divergence_from_real in G space).
__global__ void k_pot_igd(const double2* __restrict__ in, int nx, int ny, int nz, Recip9 r, int d, bool accumulate,
                          double2* __restrict__ out) {
  const long N = (long)nx * ny * nz;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < N; i += (long)gridDim.x * blockDim.x) {
    const double g = pot_gcomp(i, nx, ny, nz, r, d);
    const double2 v = in[i];
    double2 o = make_double2(-g * v.y, g * v.x);
    if (accumulate) {
      o.x += out[i].x;
      o.y += out[i].y;
    }
    out[i] = o;
  }
}

__global__ void k_pot_real_part(const double2* __restrict__ in, long N, double* __restrict__ out) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < N; i += (long)gridDim.x * blockDim.x) out[i] = in[i].x;
}

// fill_gga_xc_fields (scf/xc_fields.zig:86-106): vr = df/dn, grad_d <- df/dg2 grad_d, part = sum f.
__global__ void __launch_bounds__(kPotThreads) k_pot_pbe(const double* __restrict__ rho, long N, double* __restrict__ gx,
                                                         double* __restrict__ gy, double* __restrict__ gz,
                                                         double* __restrict__ vr, double* __restrict__ part) {
  __shared__ double red[kPotThreads / 32];
  double s = 0.0;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < N; i += (long)gridDim.x * blockDim.x) {
    const double x = gx[i], y = gy[i], z = gz[i];
    double f, vn, vg;
    pbe_point(rho[i], x * x + y * y + z * z, f, vn, vg);
    vr[i] = vn;
    gx[i] = vg * x;
    gy[i] = vg * y;
    gz[i] = vg * z;
    s += f;
  }
  s = block_sum(s, red);
  if (threadIdx.x == 0) part[blockIdx.x] = s;
}

// out = (vr - 2 Re(div)) as a complex field (compute_gga_xc_fields, xc_fields.zig:137-139).
__global__ void k_pot_gga_vxc(const double* __restrict__ vr, const double2* __restrict__ div, long N, double2* __restrict__ out) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < N; i += (long)gridDim.x * blockDim.x)
    out[i] = make_double2(vr[i] - 2.0 * div[i].x, 0.0);
}

// Local pseudopotential forces (local_pseudo_forces, forces/local_force.zig:21-80):
// F_a = sum_G 2 ff_s(|G|) G Im(e^{iG.tau_a} rho(G)) over 1e-12 < G^2 <= g2max, rho(G) = a / N.
// Grid (chunks, atoms): each block sums its chunk of G for one atom; part[(a * chunks + chunk) * 3 + d].
constexpr int kLfChunks = 64;
__global__ void __launch_bounds__(kPotThreads) k_pot_local_force(const double2* __restrict__ a, const double* __restrict__ g2,
                                                                 int nx, int ny, int nz, Recip9 r,
                                                                 LocalFF ff, const int* __restrict__ species,
                                                                 const double* __restrict__ pos, double g2max,
                                                                 double* __restrict__ part) {
  __shared__ double red[kPotThreads / 32];
  const long N = (long)nx * ny * nz;
  const int atom = blockIdx.y, chunk = blockIdx.x;
  const long per = (N + kLfChunks - 1) / kLfChunks;
  const long i0 = chunk * per, i1 = min(N, i0 + per);
  const int sp = species[atom];
  const double tx = pos[3 * atom], ty = pos[3 * atom + 1], tz = pos[3 * atom + 2];
  const double inv = 1.0 / (double)N;
  double fx = 0.0, fy = 0.0, fz = 0.0;
  for (long i = i0 + threadIdx.x; i < i1; i += blockDim.x) {
    const double q = g2[i];
    if (!ff.keep(q, g2max)) continue;
    const double gx = pot_gcomp(i, nx, ny, nz, r, 0), gy = pot_gcomp(i, nx, ny, nz, r, 1), gz = pot_gcomp(i, nx, ny, nz, r, 2);
    double sn, cs;
    sincos(gx * tx + gy * ty + gz * tz, &sn, &cs);
    const double2 rg = make_double2(a[i].x * inv, a[i].y * inv);
    const double w = ff.ry(sp, q, i) * (cs * rg.y + sn * rg.x);  // Im(e^{iG.tau} rho(G))
    fx += w * gx;
    fy += w * gy;
    fz += w * gz;
  }
  fx = block_sum(fx, red);
  fy = block_sum(fy, red);
  fz = block_sum(fz, red);
  if (threadIdx.x == 0) {
    double* o = part + ((long)atom * kLfChunks + chunk) * 3;
    o[0] = fx;
    o[1] = fy;
    o[2] = fz;
  }
}

// ---- radial projector tables (RadialTableSet, pseudopotential/nonlocal.zig:8-21, 59-71, 250-338) ----
// Spherical Bessel j_l(x): the series below 1e-6, closed forms for l <= 1, downward (Miller)
// recursion normalised by j_0 above (up to 256 terms, else the upward recurrence).
__device__ double sph_bessel(int l, double x) {
  if (fabs(x) < 1e-6) {
    const double x2 = x * x;
    if (l == 0) return 1.0 - x2 / 6.0 + x2 * x2 / 120.0;
    if (l == 1) return x / 3.0 - x * x2 / 30.0;
    if (l == 2) return x2 / 15.0 - x2 * x2 / 210.0;
    if (l == 3) return x * x2 / 105.0;
    return 0.0;
  }
  if (l == 0) return sin(x) / x;
  if (l == 1) return sin(x) / (x * x) - cos(x) / x;
  const int nm = l + 1;
  const int nlim = x < 1.0 ? nm + (int)(15.0 * x) + 1 : nm + (int)(1.36 * x) + 15;
  if (nlim > 256) {
    if (l > x + 50.0) return 0.0;
    double jlm1 = sin(x) / x, jl = sin(x) / (x * x) - cos(x) / x;
    for (int n = 1; n < l; ++n) {
      const double jlp1 = (2.0 * n + 1.0) / x * jl - jlm1;
      jlm1 = jl;
      jl = jlp1;
      if (!isfinite(jl)) return 0.0;
    }
    return jl;
  }
  const double xi = 1.0 / x;
  double up = 0.0, cur = 1.0e-18, want = 0.0;  // sb[n+1], sb[n]; nlim > l, so sb[l] is set below
  for (int n = nlim; n > 0; --n) {
    const double down = (2.0 * n + 1.0) * xi * cur - up;  // sb[n-1]
    up = cur;
    cur = down;
    if (n - 1 == nm - 1) want = cur;
  }
  return want * ((sin(x) / x) / cur);
}

// out[i] = sum_j r_j (r beta)_j j_l(q_i r_j) rab_j w_j, q_i = i * gmax / (nq - 1), w the composite
// trapezoid weights of radial_integration.zig:7-13.  One block per q point.
__global__ void __launch_bounds__(kPotThreads) k_radial_table(int l, int nr, const double* __restrict__ r,
                                                              const double* __restrict__ rbeta, const double* __restrict__ rab,
                                                              double dq, double* __restrict__ out) {
  __shared__ double red[kPotThreads / 32];
  const double q = dq * blockIdx.x;
  const double cw[5] = {23.75 / 72.0, 95.10 / 72.0, 55.20 / 72.0, 79.30 / 72.0, 70.65 / 72.0};
  double s = 0.0;
  for (int j = threadIdx.x; j < nr; j += blockDim.x) {
    double w = 1.0;
    if (nr >= 10) {
      if (j < 5) w = cw[j];
      else if (j >= nr - 5) w = cw[nr - 1 - j];
    }
    s += r[j] * rbeta[j] * sph_bessel(l, q * r[j]) * rab[j] * w;
  }
  s = block_sum(s, red);
  if (threadIdx.x == 0) out[blockIdx.x] = s;
}

// ---- density symmetrisation (symmetrize_density, scf/density_symmetry.zig:27-94) ----
// out(G) = (1/nops) sum_op in(k_rot G) e^{-2 pi i frac(G . t)}, G the signed Miller indices of the
// box (index i <-> i if i <= (n-1)/2, else i - n), the rotated G wrapped into the box, the phase
// only where frac(G . t) is more than 1e-12 from an integer.  One thread per output G; the
// operations are staged in shared memory (k_rot as 9 ints row-major, t fractional).
constexpr int kSymMaxOps = 192;  // a cubic conventional cell: 48 rotations x 4 centring translations
__device__ __forceinline__ int sym_freq(int i, int n) { return i <= (n - 1) / 2 ? i : i - n; }
__device__ __forceinline__ int sym_wrap(int g, int n) {
  const int r = g % n;
  return r < 0 ? r + n : r;
}
__global__ void __launch_bounds__(kPotThreads) k_sym_density(const double2* __restrict__ in, int nx, int ny, int nz, int nops,
                                                             const int* __restrict__ k_rot, const double* __restrict__ trans,
                                                             double2* __restrict__ out) {
  __shared__ int skr[kSymMaxOps * 9];
  __shared__ double st[kSymMaxOps * 3];
  for (int q = threadIdx.x; q < nops * 9; q += blockDim.x) skr[q] = k_rot[q];
  for (int q = threadIdx.x; q < nops * 3; q += blockDim.x) st[q] = trans[q];
  __syncthreads();
  const long N = (long)nx * ny * nz;
  const double inv = 1.0 / (double)nops;
  for (long idx = blockIdx.x * (long)blockDim.x + threadIdx.x; idx < N; idx += (long)gridDim.x * blockDim.x) {
    const int x = (int)(idx % nx), y = (int)((idx / nx) % ny), z = (int)(idx / ((long)nx * ny));
    const int h = sym_freq(x, nx), k = sym_freq(y, ny), l = sym_freq(z, nz);
    double2 sum = make_double2(0.0, 0.0);
    for (int o = 0; o < nops; ++o) {
      const int* m = skr + 9 * o;
      const int ix = sym_wrap(m[0] * h + m[1] * k + m[2] * l, nx);
      const int iy = sym_wrap(m[3] * h + m[4] * k + m[5] * l, ny);
      const int iz = sym_wrap(m[6] * h + m[7] * k + m[8] * l, nz);
      double2 term = in[ix + (long)nx * (iy + (long)ny * iz)];
      const double dot = (double)h * st[3 * o] + (double)k * st[3 * o + 1] + (double)l * st[3 * o + 2];
      const double fr = dot - floor(dot);
      if (fr > 1e-12 && fr < 1.0 - 1e-12) {
        double sn, cs;
        sincospi(-2.0 * fr, &sn, &cs);
        term = make_double2(term.x * cs - term.y * sn, term.x * sn + term.y * cs);
      }
      sum.x += term.x;
      sum.y += term.y;
    }
    out[idx] = make_double2(sum.x * inv, sum.y * inv);
  }
}

// out_r = vloc + Re(v) * N (v holds FFT^-1 / N of the G-space field).
__global__ void k_pot_real(const double2* __restrict__ v, const double* __restrict__ vloc, long N, double* __restrict__ out) {
  const double scale = (double)N;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < N; i += (long)gridDim.x * blockDim.x)
    out[i] = (vloc ? vloc[i] : 0.0) + v[i].x * scale;
}

// part[j][block] = <r_new, hist_r[j]> over the block's share, j < m.
__global__ void __launch_bounds__(kPotThreads) k_pulay_dots(const double* __restrict__ rn, const double* __restrict__ hist,
                                                            const int* __restrict__ slots, int m, long n,
                                                            double* __restrict__ part) {
  __shared__ double red[kPotThreads / 32];
  for (int j = 0; j < m; ++j) {
    const double* h = hist + (long)slots[j] * n;
    double s = 0.0;
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) s += rn[i] * h[i];
    s = block_sum(s, red);
    if (threadIdx.x == 0) part[(long)j * kPotBlocks + blockIdx.x] = s;
  }
}

// x = sum_j c_j (x_j + beta r_j) over the history slots.
__global__ void k_pulay_combine(const double* __restrict__ hx, const double* __restrict__ hr, const int* __restrict__ slots,
                                const double* __restrict__ c, int m, long n, double beta, double* __restrict__ x) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    double s = 0.0;
    for (int j = 0; j < m; ++j) {
      const long o = (long)slots[j] * n + i;
      s += c[j] * (hx[o] + beta * hr[o]);
    }
    x[i] = s;
  }
}

__global__ void k_axpy_into(const double* __restrict__ x, const double* __restrict__ r, long n, double beta,
                            double* __restrict__ out) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) out[i] = x[i] + beta * r[i];
}

// solve_pulay_system (mixing.zig:341-405): Gaussian elimination with partial pivoting on the
// bordered (m+1) x (m+1) system.  Two departures, both in the host driver too: the overlap block is
// first divided by its largest diagonal entry (the weights are unchanged; the pivot test becomes
// relative to the residual size), and a pivot below 1e-12 returns no solution, upon which the
// caller drops its oldest pair and solves again, where the reference averages the whole history
// (which stalls the mixing once more pairs are held than the residuals have directions).
std::vector<double> solve_pulay(std::vector<double> A, std::vector<double> b, int size) {
  {
    const int m = size - 1;
    double d = 0.0;
    for (int i = 0; i < m; ++i) d = std::max(d, A[i * size + i]);
    if (d > 0.0)
      for (int i = 0; i < m; ++i)
        for (int j = 0; j < m; ++j) A[i * size + j] /= d;
  }
  for (int col = 0; col < size; ++col) {
    int max_row = col;
    double max_val = std::fabs(A[col * size + col]);
    for (int row = col + 1; row < size; ++row) {
      const double v = std::fabs(A[row * size + col]);
      if (v > max_val) {
        max_val = v;
        max_row = row;
      }
    }
    if (max_row != col) {
      for (int j = 0; j < size; ++j) std::swap(A[col * size + j], A[max_row * size + j]);
      std::swap(b[col], b[max_row]);
    }
    const double pivot = A[col * size + col];
    if (std::fabs(pivot) < 1e-12) return {};  // singular: the caller drops its oldest pair
    for (int row = col + 1; row < size; ++row) {
      const double factor = A[row * size + col] / pivot;
      for (int j = col; j < size; ++j) A[row * size + j] -= factor * A[col * size + j];
      b[row] -= factor * b[col];
    }
  }
  std::vector<double> r(size);
  for (int i = size - 1; i >= 0; --i) {
    double s = b[i];
    for (int j = i + 1; j < size; ++j) s -= A[i * size + j] * r[j];
    r[i] = s / A[i * size + i];
  }
  return r;
}

}  // namespace
}  // namespace dftcuda

using namespace dftcuda;

struct dftcuda_pctx {
  int nx = 0, ny = 0, nz = 0;
  long N = 0;
  double volume = 0.0;
  double recip[9] = {};
  int history = 0;
  dftcuda_fft_plan* plan = nullptr;
  cudaStream_t stream = nullptr;
  double* g2 = nullptr;       // N
  double2* a = nullptr;       // N complex scratch
  double2* b = nullptr;       // N complex scratch
  double* rho = nullptr;      // N staging for host densities
  double2* vin = nullptr;     // N complex staging for host inputs
  double2* vout = nullptr;    // N complex staging for host outputs
  int functional = DFTCUDA_XC_LDA_PZ;
  double2* w = nullptr;       // GGA: N complex (the divergence in G space)
  double* gr = nullptr;       // GGA: 3 N real (grad n, then df/dg2 grad n)
  double* vr = nullptr;       // GGA: N real (df/dn, then V_xc)
  double* part = nullptr;     // kPotBlocks x max(2, history) partial sums
  double* h_part = nullptr;   // pinned host copy
  // Pulay history: `history` slots of n doubles each for inputs and residuals, plus staging
  long pn = 0;                // vector length the history holds (0 until the first mix)
  double* hx = nullptr;
  double* hr = nullptr;
  double* px = nullptr;       // n staging (x in / out)
  double* pr = nullptr;       // n staging (residual)
  int* d_slots = nullptr;
  double* d_coef = nullptr;
  int* sym_kr = nullptr;      // symmetry operations (kSymMaxOps x 9 ints, x 3 doubles), on first use
  double* sym_t = nullptr;
  std::vector<int> order;     // slots oldest first
  std::vector<double> B;      // history x history residual overlaps, by slot
};

static int pctx_fail_free(dftcuda_pctx* c, int status) {
  dftcuda_pctx_destroy(c);
  return status;
}

extern "C" int dftcuda_pctx_create(dftcuda_pctx** out, int nx, int ny, int nz, double volume, const double* recip,
                                   int pulay_history) {
  if (!out || nx <= 0 || ny <= 0 || nz <= 0 || !(volume > 0.0) || !recip || pulay_history < 0 || pulay_history > 64)
    return fail(DFTCUDA_ERR_INVALID_ARGUMENT, "pctx_create: bad arguments (history must be 0..64)");
  *out = nullptr;
  auto* c = new dftcuda_pctx();
  c->nx = nx; c->ny = ny; c->nz = nz;
  c->N = (long)nx * ny * nz;
  c->volume = volume;
  for (int i = 0; i < 9; ++i) c->recip[i] = recip[i];
  c->history = pulay_history;
  int st = dftcuda_fft_plan_create(&c->plan, nx, ny, nz);
  if (st != DFTCUDA_OK) return pctx_fail_free(c, st);
  const long N = c->N;
  const int nparts = std::max(2, pulay_history);
  if (cudaStreamCreateWithFlags(&c->stream, cudaStreamDefault) != cudaSuccess ||
      dev_malloc(&c->g2, sizeof(double) * N) != cudaSuccess || dev_malloc(&c->a, sizeof(double2) * N) != cudaSuccess ||
      dev_malloc(&c->b, sizeof(double2) * N) != cudaSuccess || dev_malloc(&c->rho, sizeof(double) * N) != cudaSuccess ||
      dev_malloc(&c->vin, sizeof(double2) * N) != cudaSuccess || dev_malloc(&c->vout, sizeof(double2) * N) != cudaSuccess ||
      dev_malloc(&c->part, sizeof(double) * kPotBlocks * nparts) != cudaSuccess ||
      cudaMallocHost(&c->h_part, sizeof(double) * kPotBlocks * nparts) != cudaSuccess ||
      dev_malloc(&c->d_slots, sizeof(int) * 64) != cudaSuccess || dev_malloc(&c->d_coef, sizeof(double) * 65) != cudaSuccess)
    return pctx_fail_free(c, fail(DFTCUDA_ERR_CUDA, "pctx_create: device allocation failed"));
  const double* r = recip;
  k_pot_g2<<<kPotBlocks, kPotThreads, 0, c->stream>>>(nx, ny, nz, r[0], r[1], r[2], r[3], r[4], r[5], r[6], r[7], r[8], c->g2);
  count_launch();
  if (cudaStreamSynchronize(c->stream) != cudaSuccess) return pctx_fail_free(c, fail(DFTCUDA_ERR_CUDA, "pctx_create: G^2"));
  *out = c;
  return DFTCUDA_OK;
}

extern "C" int dftcuda_pctx_destroy(dftcuda_pctx* c) {
  if (!c) return DFTCUDA_OK;
  if (c->stream) cudaStreamSynchronize(c->stream);
  for (void* p : {(void*)c->w, (void*)c->gr, (void*)c->vr})
    if (p) cudaFree(p);
  for (void* p : {(void*)c->g2, (void*)c->a, (void*)c->b, (void*)c->rho, (void*)c->vin, (void*)c->vout, (void*)c->part, (void*)c->hx,
                  (void*)c->hr, (void*)c->px, (void*)c->pr, (void*)c->d_slots, (void*)c->d_coef, (void*)c->sym_kr,
                  (void*)c->sym_t})
    if (p) cudaFree(p);
  if (c->h_part) cudaFreeHost(c->h_part);
  if (c->plan) dftcuda_fft_plan_destroy(c->plan);
  if (c->stream) cudaStreamDestroy(c->stream);
  delete c;
  return DFTCUDA_OK;
}

// A device view of n bytes of `src` (host or device): device pointers pass through, host data is
// copied into `staging`.
static const void* device_view(const void* src, void* staging, size_t bytes, cudaStream_t s, int* st) {
  if (is_device_pointer(src)) return src;
  if (cudaMemcpyAsync(staging, src, bytes, cudaMemcpyHostToDevice, s) != cudaSuccess)
    *st = fail(DFTCUDA_ERR_CUDA, "potential: host-to-device copy failed");
  return staging;
}

static int copy_out(void* dst, const void* src, size_t bytes, cudaStream_t s) {
  DFT_CUDA_TRY(cudaMemcpyAsync(dst, src, bytes, is_device_pointer(dst) ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, s));
  return DFTCUDA_OK;
}

extern "C" int dftcuda_pctx_set_functional(dftcuda_pctx* c, int functional) {
  if (!c || (functional != DFTCUDA_XC_LDA_PZ && functional != DFTCUDA_XC_PBE))
    return fail(DFTCUDA_ERR_INVALID_ARGUMENT, "pctx_set_functional: LDA-PZ (0) or PBE (1)");
  if (functional == DFTCUDA_XC_PBE && !c->w) {
    const long N = c->N;
    if (dev_malloc(&c->w, sizeof(double2) * N) != cudaSuccess || dev_malloc(&c->gr, sizeof(double) * 3 * N) != cudaSuccess ||
        dev_malloc(&c->vr, sizeof(double) * N) != cudaSuccess) {
      for (void** p : {(void**)&c->w, (void**)&c->gr, (void**)&c->vr})
        if (*p) {
          cudaFree(*p);
          *p = nullptr;
        }
      return fail(DFTCUDA_ERR_CUDA, "pctx_set_functional: GGA buffers");
    }
  }
  c->functional = functional;
  return DFTCUDA_OK;
}

// compute_gga_xc_fields (scf/xc_fields.zig:108-142) on the device: grad n from three inverse FFTs of
// i G rho(G); the point functional; the divergence of df/dg2 grad n from three forward FFTs and one
// inverse; V_xc = df/dn - 2 div back to G space in b (N V_xc(G), unnormalised).  On entry a holds
// N rho(G); returns the sum of f over the grid.
static int gga_vxc(dftcuda_pctx* c, const double* rho, double* exc_sum) {
  const long N = c->N;
  cudaStream_t s = c->stream;
  Recip9 r;
  for (int i = 0; i < 9; ++i) r.b[i] = c->recip[i];
  for (int d = 0; d < 3; ++d) {
    k_pot_igd<<<kPotBlocks, kPotThreads, 0, s>>>(c->a, c->nx, c->ny, c->nz, r, d, false, c->b);
    count_launch();
    DFT_TRY(fft3d_on_stream(c->plan, c->b, +1, s));
    k_pot_real_part<<<kPotBlocks, kPotThreads, 0, s>>>(c->b, N, c->gr + (long)d * N);
    count_launch();
  }
  k_pot_pbe<<<kPotBlocks, kPotThreads, 0, s>>>(rho, N, c->gr, c->gr + N, c->gr + 2 * N, c->vr, c->part);
  count_launch();
  DFT_CUDA_TRY(cudaMemcpyAsync(c->h_part, c->part, sizeof(double) * kPotBlocks, cudaMemcpyDeviceToHost, s));
  for (int d = 0; d < 3; ++d) {
    k_pot_to_complex<<<kPotBlocks, kPotThreads, 0, s>>>(c->gr + (long)d * N, N, c->b);
    count_launch();
    DFT_TRY(fft3d_on_stream(c->plan, c->b, -1, s));
    k_pot_igd<<<kPotBlocks, kPotThreads, 0, s>>>(c->b, c->nx, c->ny, c->nz, r, d, d > 0, c->w);
    count_launch();
  }
  DFT_TRY(fft3d_on_stream(c->plan, c->w, +1, s));  // div(r) = (1/N) sum_G i G . B(G) e^{iGr}
  k_pot_gga_vxc<<<kPotBlocks, kPotThreads, 0, s>>>(c->vr, c->w, N, c->b);
  count_launch();
  DFT_TRY(fft3d_on_stream(c->plan, c->b, -1, s));
  DFT_CUDA_TRY(cudaStreamSynchronize(s));
  double e = 0.0;
  for (int i = 0; i < kPotBlocks; ++i) e += c->h_part[i];
  *exc_sum = e;
  return DFTCUDA_OK;
}

extern "C" int dftcuda_hxc_potential(dftcuda_pctx* c, const double* rho_r, const double* v_in_g, double* v_out_g,
                                     dftcuda_hxc_terms* terms) {
  if (!c || !rho_r || !v_out_g) return fail(DFTCUDA_ERR_INVALID_ARGUMENT, "hxc_potential: null argument");
  const long N = c->N;
  cudaStream_t s = c->stream;
  int st = DFTCUDA_OK;
  const double* rho = (const double*)device_view(rho_r, c->rho, sizeof(double) * N, s, &st);
  const double2* vin = v_in_g ? (const double2*)device_view(v_in_g, c->vin, sizeof(double2) * N, s, &st) : nullptr;
  if (st != DFTCUDA_OK) return st;
  double exc = 0.0;
  if (c->functional == DFTCUDA_XC_PBE) {
    k_pot_to_complex<<<kPotBlocks, kPotThreads, 0, s>>>(rho, N, c->a);
    count_launch();
    DFT_TRY(fft3d_on_stream(c->plan, c->a, -1, s));
    DFT_TRY(gga_vxc(c, rho, &exc));
  } else {
    k_pot_xc<<<kPotBlocks, kPotThreads, 0, s>>>(rho, N, c->a, c->b, c->part);
    count_launch();
    DFT_CUDA_TRY(cudaMemcpyAsync(c->h_part, c->part, sizeof(double) * kPotBlocks, cudaMemcpyDeviceToHost, s));
    DFT_CUDA_TRY(cudaStreamSynchronize(s));
    for (int i = 0; i < kPotBlocks; ++i) exc += c->h_part[i];
    DFT_TRY(fft3d_on_stream(c->plan, c->a, -1, s));
    DFT_TRY(fft3d_on_stream(c->plan, c->b, -1, s));
  }
  double2* out = is_device_pointer(v_out_g) ? (double2*)v_out_g : c->vout;
  k_pot_hartree<<<kPotBlocks, kPotThreads, 0, s>>>(c->a, c->b, c->g2, N, vin, out, c->part);
  count_launch();
  if (out != (double2*)v_out_g) DFT_TRY(copy_out(v_out_g, out, sizeof(double2) * N, s));
  DFT_CUDA_TRY(cudaMemcpyAsync(c->h_part, c->part, sizeof(double) * 2 * kPotBlocks, cudaMemcpyDeviceToHost, s));
  DFT_CUDA_TRY(cudaStreamSynchronize(s));
  double eh = 0.0, ei = 0.0;
  for (int i = 0; i < kPotBlocks; ++i) {
    eh += c->h_part[i];
    ei += c->h_part[kPotBlocks + i];
  }
  if (terms) {
    terms->e_hartree = 0.5 * c->volume * eh;
    terms->e_xc = exc * c->volume / (double)N;
    terms->int_vin_rho = v_in_g ? c->volume * ei : 0.0;
  }
  return DFTCUDA_OK;
}

extern "C" int dftcuda_potential_real(dftcuda_pctx* c, const double* v_g, const double* vloc_r, double* out_r) {
  if (!c || !v_g || !out_r) return fail(DFTCUDA_ERR_INVALID_ARGUMENT, "potential_real: null argument");
  const long N = c->N;
  cudaStream_t s = c->stream;
  DFT_CUDA_TRY(cudaMemcpyAsync(c->a, v_g, sizeof(double2) * N,
                               is_device_pointer(v_g) ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, s));
  int st = DFTCUDA_OK;
  const double* vloc = vloc_r ? (const double*)device_view(vloc_r, c->rho, sizeof(double) * N, s, &st) : nullptr;
  if (st != DFTCUDA_OK) return st;
  DFT_TRY(fft3d_on_stream(c->plan, c->a, +1, s));
  double* out = is_device_pointer(out_r) ? out_r : reinterpret_cast<double*>(c->b);
  k_pot_real<<<kPotBlocks, kPotThreads, 0, s>>>(c->a, vloc, N, out);
  count_launch();
  if (out != out_r) DFT_TRY(copy_out(out_r, out, sizeof(double) * N, s));
  DFT_CUDA_TRY(cudaStreamSynchronize(s));
  return DFTCUDA_OK;
}

extern "C" int dftcuda_symmetrize_density(dftcuda_pctx* c, int nops, const int* k_rot, const double* trans, double* rho_r) {
  if (!c || !rho_r || nops < 0 || nops > kSymMaxOps || (nops > 1 && (!k_rot || !trans)))
    return fail(DFTCUDA_ERR_INVALID_ARGUMENT, "symmetrize_density: bad arguments (0..192 operations)");
  if (nops <= 1) return DFTCUDA_OK;  // the identity alone leaves the density as it is
  for (int q = 0; q < 3 * nops; ++q)
    if (!std::isfinite(trans[q])) return fail(DFTCUDA_ERR_INVALID_ARGUMENT, "symmetrize_density: non-finite translation");
  const long N = c->N;
  cudaStream_t s = c->stream;
  if (!c->sym_kr) {
    if (dev_malloc(&c->sym_kr, sizeof(int) * 9 * kSymMaxOps) != cudaSuccess ||
        dev_malloc(&c->sym_t, sizeof(double) * 3 * kSymMaxOps) != cudaSuccess)
      return fail(DFTCUDA_ERR_CUDA, "symmetrize_density: allocation failed");
  }
  DFT_CUDA_TRY(cudaMemcpyAsync(c->sym_kr, k_rot, sizeof(int) * 9 * nops, cudaMemcpyDefault, s));
  DFT_CUDA_TRY(cudaMemcpyAsync(c->sym_t, trans, sizeof(double) * 3 * nops, cudaMemcpyDefault, s));
  int st = DFTCUDA_OK;
  const double* rho = (const double*)device_view(rho_r, c->rho, sizeof(double) * N, s, &st);
  if (st != DFTCUDA_OK) return st;
  k_pot_to_complex<<<kPotBlocks, kPotThreads, 0, s>>>(rho, N, c->a);
  count_launch();
  DFT_TRY(fft3d_on_stream(c->plan, c->a, -1, s));
  k_sym_density<<<kPotBlocks, kPotThreads, 0, s>>>(c->a, c->nx, c->ny, c->nz, nops, c->sym_kr, c->sym_t, c->b);
  count_launch();
  DFT_TRY(fft3d_on_stream(c->plan, c->b, +1, s));
  double* out = is_device_pointer(rho_r) ? rho_r : c->rho;
  k_pot_real_part<<<kPotBlocks, kPotThreads, 0, s>>>(c->b, N, out);
  count_launch();
  if (out != rho_r) DFT_TRY(copy_out(rho_r, out, sizeof(double) * N, s));
  DFT_CUDA_TRY(cudaStreamSynchronize(s));
  return DFTCUDA_OK;
}

// The species form factors of the ionic-potential and local-force calls: the 6 GTH parameters per
// species (gth), or each species' radial mesh (mesh_off[nspecies + 1] into r, rab, vloc; z[nspecies]),
// whose form factor k_pot_vq_radial evaluates at every box point.
struct FFArgs {
  const double* gth = nullptr;
  const size_t* mesh_off = nullptr;
  const double *r = nullptr, *rab = nullptr, *vloc = nullptr, *z = nullptr;
};

// Device copies of the form-factor inputs and, for radial meshes, the per-point form factors.
struct FFDevice {
  double* buf = nullptr;
  int* off = nullptr;
  LocalFF ff;
  ~FFDevice() {
    if (buf) cudaFree(buf);
    if (off) cudaFree(off);
  }
  int init(const FFArgs& a, int nspecies, const double* g2, long N, cudaStream_t s) {
    if (a.gth) {
      if (dev_malloc(&buf, sizeof(double) * 6 * nspecies) != cudaSuccess) return fail(DFTCUDA_ERR_CUDA, "form factors: allocation failed");
      DFT_CUDA_TRY(cudaMemcpyAsync(buf, a.gth, sizeof(double) * 6 * nspecies, cudaMemcpyDefault, s));
      ff.gth = buf;
      return DFTCUDA_OK;
    }
    std::vector<int> ho(nspecies + 1);
    for (int i = 0; i <= nspecies; ++i) {
      if (a.mesh_off[i] > (size_t)INT32_MAX || (i > 0 && a.mesh_off[i] < a.mesh_off[i - 1]))
        return fail(DFTCUDA_ERR_INVALID_ARGUMENT, "radial form factors: mesh offsets must ascend");
      ho[i] = (int)a.mesh_off[i];
    }
    const size_t nr = (size_t)ho[nspecies] - ho[0];
    if (ho[0] != 0 || nr == 0) return fail(DFTCUDA_ERR_INVALID_ARGUMENT, "radial form factors: empty mesh");
    if (dev_malloc(&buf, sizeof(double) * (3 * nr + nspecies + (size_t)nspecies * N)) != cudaSuccess ||
        dev_malloc(&off, sizeof(int) * (nspecies + 1)) != cudaSuccess)
      return fail(DFTCUDA_ERR_OUT_OF_MEMORY, "radial form factors: allocation failed");
    double *dr = buf, *drab = buf + nr, *dv = buf + 2 * nr, *dz = buf + 3 * nr, *vq = dz + nspecies;
    DFT_CUDA_TRY(cudaMemcpyAsync(dr, a.r, sizeof(double) * nr, cudaMemcpyDefault, s));
    DFT_CUDA_TRY(cudaMemcpyAsync(drab, a.rab, sizeof(double) * nr, cudaMemcpyDefault, s));
    DFT_CUDA_TRY(cudaMemcpyAsync(dv, a.vloc, sizeof(double) * nr, cudaMemcpyDefault, s));
    DFT_CUDA_TRY(cudaMemcpyAsync(dz, a.z, sizeof(double) * nspecies, cudaMemcpyDefault, s));
    DFT_CUDA_TRY(cudaMemcpyAsync(off, ho.data(), sizeof(int) * (nspecies + 1), cudaMemcpyHostToDevice, s));
    k_pot_vq_radial<<<(unsigned)std::min<long>(ceil_div(N, kPotThreads), 65535), kPotThreads, 0, s>>>(g2, N, nspecies, off, dr, drab, dv,
                                                                                                      dz, vq);
    count_launch();
    DFT_CUDA_TRY(cudaGetLastError());
    DFT_CUDA_TRY(cudaStreamSynchronize(s));  // ho goes out of scope
    ff.vq = vq;
    ff.N = N;
    return DFTCUDA_OK;
  }
};

static int ionic_impl(dftcuda_pctx* c, int nspecies, const FFArgs& ffa, int natoms, const int* atom_species, const double* positions,
                      double g2max, double* v_out_g, double* vloc_r) {
  if (!c || nspecies < 1 || nspecies > kIonMaxSpecies || natoms < 0 || (natoms > 0 && (!atom_species || !positions)))
    return fail(DFTCUDA_ERR_INVALID_ARGUMENT, "ionic_potential: bad arguments (1..8 species)");
  for (int a = 0; a < natoms; ++a)
    if (atom_species[a] < 0 || atom_species[a] >= nspecies)
      return fail(DFTCUDA_ERR_INVALID_ARGUMENT, "ionic_potential: atom species index out of range");
  const long N = c->N;
  cudaStream_t s = c->stream;
  double* d_pos = nullptr;
  int* d_sp = nullptr;
  auto cleanup = [&] {
    if (d_pos) cudaFree(d_pos);
    if (d_sp) cudaFree(d_sp);
  };
  FFDevice ffd;
  DFT_TRY(ffd.init(ffa, nspecies, c->g2, N, s));
  if (dev_malloc(&d_pos, sizeof(double) * 3 * std::max(natoms, 1)) != cudaSuccess ||
      dev_malloc(&d_sp, sizeof(int) * std::max(natoms, 1)) != cudaSuccess) {
    cleanup();
    return fail(DFTCUDA_ERR_CUDA, "ionic_potential: allocation failed");
  }
  int st = DFTCUDA_OK;
  if ((natoms > 0 && (cudaMemcpyAsync(d_pos, positions, sizeof(double) * 3 * natoms, cudaMemcpyDefault, s) != cudaSuccess ||
                      cudaMemcpyAsync(d_sp, atom_species, sizeof(int) * natoms, cudaMemcpyDefault, s) != cudaSuccess)))
    st = fail(DFTCUDA_ERR_CUDA, "ionic_potential: copy failed");
  if (st == DFTCUDA_OK) {
    const double* r = c->recip;
    k_pot_ionic<<<(unsigned)ceil_div(N, kPotThreads), kPotThreads, 0, s>>>(
        c->g2, c->nx, c->ny, c->nz, r[0], r[1], r[2], r[3], r[4], r[5], r[6], r[7], r[8], nspecies, ffd.ff, natoms, d_sp, d_pos,
        g2max > 0.0 ? g2max : 1e300, 1.0 / c->volume, c->b);
    count_launch();
    if (v_out_g && copy_out(v_out_g, c->b, sizeof(double2) * N, s) != DFTCUDA_OK) st = DFTCUDA_ERR_CUDA;
  }
  if (st == DFTCUDA_OK && vloc_r) {
    DFT_CUDA_TRY(cudaMemcpyAsync(c->a, c->b, sizeof(double2) * N, cudaMemcpyDeviceToDevice, s));
    st = fft3d_on_stream(c->plan, c->a, +1, s);
    if (st == DFTCUDA_OK) {
      double* out = is_device_pointer(vloc_r) ? vloc_r : reinterpret_cast<double*>(c->b);
      k_pot_real<<<kPotBlocks, kPotThreads, 0, s>>>(c->a, nullptr, N, out);
      count_launch();
      if (out != vloc_r) st = copy_out(vloc_r, out, sizeof(double) * N, s);
    }
  }
  if (cudaStreamSynchronize(s) != cudaSuccess && st == DFTCUDA_OK) st = fail(DFTCUDA_ERR_CUDA, "ionic_potential: kernel failed");
  cleanup();
  return st;
}

static int local_forces_impl(dftcuda_pctx* c, int nspecies, const FFArgs& ffa, int natoms, const int* atom_species,
                             const double* positions, double g2max, const double* rho_r, double* forces) {
  if (!c || nspecies < 1 || natoms < 1 || !atom_species || !positions || !rho_r || !forces)
    return fail(DFTCUDA_ERR_INVALID_ARGUMENT, "local_forces: bad arguments");
  for (int a = 0; a < natoms; ++a)
    if (atom_species[a] < 0 || atom_species[a] >= nspecies)
      return fail(DFTCUDA_ERR_INVALID_ARGUMENT, "local_forces: atom species index out of range");
  const long N = c->N;
  cudaStream_t s = c->stream;
  int st = DFTCUDA_OK;
  const double* rho = (const double*)device_view(rho_r, c->rho, sizeof(double) * N, s, &st);
  if (st != DFTCUDA_OK) return st;
  double* d_pos = nullptr;
  int* d_sp = nullptr;
  double* d_part = nullptr;
  auto cleanup = [&] {
    for (void* p : {(void*)d_pos, (void*)d_sp, (void*)d_part})
      if (p) cudaFree(p);
  };
  const size_t npart = (size_t)natoms * kLfChunks * 3;
  FFDevice ffd;
  DFT_TRY(ffd.init(ffa, nspecies, c->g2, N, s));
  if (dev_malloc(&d_pos, sizeof(double) * 3 * natoms) != cudaSuccess ||
      dev_malloc(&d_sp, sizeof(int) * natoms) != cudaSuccess || dev_malloc(&d_part, sizeof(double) * npart) != cudaSuccess) {
    cleanup();
    return fail(DFTCUDA_ERR_CUDA, "local_forces: allocation failed");
  }
  std::vector<double> hp(npart);
  auto run = [&]() -> int {
    DFT_CUDA_TRY(cudaMemcpyAsync(d_pos, positions, sizeof(double) * 3 * natoms, cudaMemcpyDefault, s));
    DFT_CUDA_TRY(cudaMemcpyAsync(d_sp, atom_species, sizeof(int) * natoms, cudaMemcpyDefault, s));
    k_pot_to_complex<<<kPotBlocks, kPotThreads, 0, s>>>(rho, N, c->a);
    count_launch();
    DFT_TRY(fft3d_on_stream(c->plan, c->a, -1, s));
    Recip9 r;
    for (int i = 0; i < 9; ++i) r.b[i] = c->recip[i];
    k_pot_local_force<<<dim3(kLfChunks, natoms), kPotThreads, 0, s>>>(c->a, c->g2, c->nx, c->ny, c->nz, r, ffd.ff, d_sp, d_pos,
                                                                       g2max > 0.0 ? g2max : 1e300, d_part);
    count_launch();
    DFT_CUDA_TRY(cudaMemcpyAsync(hp.data(), d_part, sizeof(double) * npart, cudaMemcpyDeviceToHost, s));
    DFT_CUDA_TRY(cudaStreamSynchronize(s));
    std::vector<double> f(3 * (size_t)natoms, 0.0);
    for (int a = 0; a < natoms; ++a)
      for (int ch = 0; ch < kLfChunks; ++ch)
        for (int d = 0; d < 3; ++d) f[3 * a + d] += hp[((size_t)a * kLfChunks + ch) * 3 + d];
    if (is_device_pointer(forces)) DFT_CUDA_TRY(cudaMemcpy(forces, f.data(), sizeof(double) * f.size(), cudaMemcpyHostToDevice));
    else std::memcpy(forces, f.data(), sizeof(double) * f.size());
    return DFTCUDA_OK;
  };
  st = run();
  cleanup();
  return st;
}

extern "C" int dftcuda_ionic_potential(dftcuda_pctx* c, int nspecies, const double* gth, int natoms, const int* atom_species,
                                       const double* positions, double g2max, double* v_out_g, double* vloc_r) {
  if (!gth) return fail(DFTCUDA_ERR_INVALID_ARGUMENT, "ionic_potential: null parameters");
  FFArgs f;
  f.gth = gth;
  return ionic_impl(c, nspecies, f, natoms, atom_species, positions, g2max, v_out_g, vloc_r);
}

extern "C" int dftcuda_ionic_potential_radial(dftcuda_pctx* c, int nspecies, const size_t* mesh_off, const double* r,
                                              const double* rab, const double* vloc, const double* z_valence, int natoms,
                                              const int* atom_species, const double* positions, double g2max, double* v_out_g,
                                              double* vloc_r) {
  if (!mesh_off || !r || !rab || !vloc || !z_valence) return fail(DFTCUDA_ERR_INVALID_ARGUMENT, "ionic_potential_radial: null mesh");
  FFArgs f;
  f.mesh_off = mesh_off;
  f.r = r;
  f.rab = rab;
  f.vloc = vloc;
  f.z = z_valence;
  return ionic_impl(c, nspecies, f, natoms, atom_species, positions, g2max, v_out_g, vloc_r);
}

extern "C" int dftcuda_local_forces(dftcuda_pctx* c, int nspecies, const double* gth, int natoms, const int* atom_species,
                                    const double* positions, double g2max, const double* rho_r, double* forces) {
  if (!gth) return fail(DFTCUDA_ERR_INVALID_ARGUMENT, "local_forces: null parameters");
  FFArgs f;
  f.gth = gth;
  return local_forces_impl(c, nspecies, f, natoms, atom_species, positions, g2max, rho_r, forces);
}

extern "C" int dftcuda_local_forces_radial(dftcuda_pctx* c, int nspecies, const size_t* mesh_off, const double* r,
                                           const double* rab, const double* vloc, const double* z_valence, int natoms,
                                           const int* atom_species, const double* positions, double g2max, const double* rho_r,
                                           double* forces) {
  if (!mesh_off || !r || !rab || !vloc || !z_valence) return fail(DFTCUDA_ERR_INVALID_ARGUMENT, "local_forces_radial: null mesh");
  FFArgs f;
  f.mesh_off = mesh_off;
  f.r = r;
  f.rab = rab;
  f.vloc = vloc;
  f.z = z_valence;
  return local_forces_impl(c, nspecies, f, natoms, atom_species, positions, g2max, rho_r, forces);
}

extern "C" int dftcuda_radial_table(int l, size_t nr, const double* r, const double* rbeta, const double* rab, size_t nq,
                                    double gmax, double* out) {
  if (l < 0 || nr == 0 || nq < 2 || !r || !rbeta || !rab || !out || !(gmax > 0.0) || nr > (size_t)INT32_MAX || nq > 65535)
    return fail(DFTCUDA_ERR_INVALID_ARGUMENT, "radial_table: bad arguments (nq 2..65535)");
  double* d = nullptr;
  const size_t bytes = sizeof(double) * (3 * nr + nq);
  if (dev_malloc(&d, bytes) != cudaSuccess) return fail(DFTCUDA_ERR_CUDA, "radial_table: allocation failed");
  cudaStream_t s = nullptr;
  int st = DFTCUDA_OK;
  auto run = [&]() -> int {
    DFT_CUDA_TRY(cudaStreamCreateWithFlags(&s, cudaStreamDefault));
    DFT_CUDA_TRY(cudaMemcpyAsync(d, r, sizeof(double) * nr, cudaMemcpyDefault, s));
    DFT_CUDA_TRY(cudaMemcpyAsync(d + nr, rbeta, sizeof(double) * nr, cudaMemcpyDefault, s));
    DFT_CUDA_TRY(cudaMemcpyAsync(d + 2 * nr, rab, sizeof(double) * nr, cudaMemcpyDefault, s));
    k_radial_table<<<(unsigned)nq, kPotThreads, 0, s>>>(l, (int)nr, d, d + nr, d + 2 * nr, gmax / (double)(nq - 1), d + 3 * nr);
    count_launch();
    DFT_CUDA_TRY(cudaMemcpyAsync(out, d + 3 * nr, sizeof(double) * nq, cudaMemcpyDefault, s));
    DFT_CUDA_TRY(cudaStreamSynchronize(s));
    return DFTCUDA_OK;
  };
  st = run();
  if (s) cudaStreamDestroy(s);
  cudaFree(d);
  return st;
}

extern "C" int dftcuda_pulay_reset(dftcuda_pctx* c) {
  if (!c) return fail(DFTCUDA_ERR_INVALID_ARGUMENT, "pulay_reset: null context");
  c->order.clear();
  return DFTCUDA_OK;
}

extern "C" int dftcuda_pulay_mix(dftcuda_pctx* c, double* x, const double* residual, size_t n, double beta) {
  if (!c || !x || !residual || n == 0) return fail(DFTCUDA_ERR_INVALID_ARGUMENT, "pulay_mix: bad arguments");
  if (c->history < 1) return fail(DFTCUDA_ERR_INVALID_ARGUMENT, "pulay_mix: the context was created without history");
  cudaStream_t s = c->stream;
  const int H = c->history;
  if (c->pn != (long)n) {
    // (re)size the history for this vector length
    for (double** p : {&c->hx, &c->hr, &c->px, &c->pr})
      if (*p) {
        cudaFree(*p);
        *p = nullptr;
      }
    if (dev_malloc(&c->hx, sizeof(double) * n * H) != cudaSuccess || dev_malloc(&c->hr, sizeof(double) * n * H) != cudaSuccess ||
        dev_malloc(&c->px, sizeof(double) * n) != cudaSuccess || dev_malloc(&c->pr, sizeof(double) * n) != cudaSuccess) {
      c->pn = 0;
      return fail(DFTCUDA_ERR_CUDA, "pulay_mix: history allocation failed");
    }
    c->pn = (long)n;
    c->order.clear();
    c->B.assign((size_t)H * H, 0.0);
  }
  // the new pair goes into the oldest slot once the history is full (mix_with_residual appends,
  // then drops the oldest beyond `history`)
  int slot;
  if ((int)c->order.size() < H) {
    std::vector<bool> used(H, false);
    for (int o : c->order) used[o] = true;
    slot = 0;
    while (used[slot]) ++slot;
  } else {
    slot = c->order.front();
    c->order.erase(c->order.begin());
  }
  c->order.push_back(slot);
  DFT_CUDA_TRY(cudaMemcpyAsync(c->hx + (long)slot * n, x, sizeof(double) * n,
                               is_device_pointer(x) ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, s));
  DFT_CUDA_TRY(cudaMemcpyAsync(c->hr + (long)slot * n, residual, sizeof(double) * n,
                               is_device_pointer(residual) ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, s));
  double* xo = is_device_pointer(x) ? x : c->px;
  const int m = (int)c->order.size();
  // overlaps of the new residual with every residual held, itself included (every call, so the
  // overlap table is complete when the history first reaches two pairs)
  DFT_CUDA_TRY(cudaMemcpyAsync(c->d_slots, c->order.data(), sizeof(int) * m, cudaMemcpyHostToDevice, s));
  k_pulay_dots<<<kPotBlocks, kPotThreads, 0, s>>>(c->hr + (long)slot * n, c->hr, c->d_slots, m, (long)n, c->part);
  count_launch();
  DFT_CUDA_TRY(cudaMemcpyAsync(c->h_part, c->part, sizeof(double) * kPotBlocks * m, cudaMemcpyDeviceToHost, s));
  DFT_CUDA_TRY(cudaStreamSynchronize(s));
  for (int j = 0; j < m; ++j) {
    double d = 0.0;
    for (int i = 0; i < kPotBlocks; ++i) d += c->h_part[(long)j * kPotBlocks + i];
    c->B[(size_t)slot * H + c->order[j]] = d;
    c->B[(size_t)c->order[j] * H + slot] = d;
  }
  // DIIS weights over the newest k pairs, k from m down to 2 while the system is singular
  std::vector<double> coef;
  int first = 0;
  for (; m - first >= 2; ++first) {
    const int k = m - first, sz = k + 1;
    std::vector<double> A((size_t)sz * sz, 0.0), rhs(sz, 0.0);
    for (int i = 0; i < k; ++i) {
      for (int j = 0; j < k; ++j) A[(size_t)i * sz + j] = c->B[(size_t)c->order[first + i] * H + c->order[first + j]];
      A[(size_t)i * sz + k] = -1.0;
      A[(size_t)k * sz + i] = -1.0;
    }
    rhs[k] = -1.0;
    coef = solve_pulay(A, rhs, sz);
    if (!coef.empty()) break;
  }
  if (coef.empty()) {
    k_axpy_into<<<kPotBlocks, kPotThreads, 0, s>>>(c->hx + (long)slot * n, c->hr + (long)slot * n, (long)n, beta, xo);
    count_launch();
  } else {
    const int k = m - first;
    DFT_CUDA_TRY(cudaMemcpyAsync(c->d_slots, c->order.data() + first, sizeof(int) * k, cudaMemcpyHostToDevice, s));
    DFT_CUDA_TRY(cudaMemcpyAsync(c->d_coef, coef.data(), sizeof(double) * k, cudaMemcpyHostToDevice, s));
    k_pulay_combine<<<kPotBlocks, kPotThreads, 0, s>>>(c->hx, c->hr, c->d_slots, c->d_coef, k, (long)n, beta, xo);
    count_launch();
  }
  if (xo != x) DFT_CUDA_TRY(cudaMemcpyAsync(x, xo, sizeof(double) * n, cudaMemcpyDeviceToHost, s));
  DFT_CUDA_TRY(cudaStreamSynchronize(s));
  DFT_CUDA_TRY(cudaGetLastError());
  return DFTCUDA_OK;
}
