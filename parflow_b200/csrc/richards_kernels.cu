// Richards residual, analytic Jacobian assembly and stencil matvec.
//
// Gather form: every cell computes the fluxes (or flux derivatives) of its
// own six faces; a face shared by two cells is evaluated by both with the
// same operands in the same order, so both see identical bits and no atomics
// are needed.  Per-cell relative permeabilities are produced by a first pass
// (k_vg_all) so that each cell's van Genuchten state is evaluated once per
// iterate and shared by the residual and the Jacobian.
#include "pfgpu_device.cuh"
#include "pdl.cuh"
#include "pfgpu_kernels.h"

namespace pfgpu {

// (i, j, k) of a thread in a 3-D launch (x across the block's threads,
// rows in y, one plane per blockIdx.z): no integer division
__device__ __forceinline__ bool launch_ijk(int nx, int ny, int nz, int &i, int &j, int &k) {
  i = blockIdx.x * blockDim.x + threadIdx.x;
  j = blockIdx.y * blockDim.y + threadIdx.y;
  k = blockIdx.z;
  return i < nx && j < ny && k < nz;
}

// Van Genuchten state of every cell at one pressure iterate: kr, dkr/dp, S,
// dS/dp (problem_phase_rel_perm.c:1312-1361, problem_saturation.c:342-412).
// The residual uses kr and S; the Jacobian at the same iterate reuses all four.
// Launch bounds: these FP64 kernels are latency-bound at the occupancy their
// natural register use allows; capping registers (a few spilled bytes stay in
// L1) for 5 (8) resident blocks per SM cuts their time by about 30%.
__global__ void __launch_bounds__(256, 5) k_vg_all(DevProblem P, const double *__restrict__ p, double *__restrict__ kr,
                         double *__restrict__ dkr, double *__restrict__ sat,
                         double *__restrict__ dsat) {
  pdl_enter();
  long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (c >= P.n) return;
  VGAll v = vg_all(P, p[c], vg_at(P, c));
  if (P.krt) {  // relative permeability from the lookup table
    const double pc = p[c];
    if (pc >= 0.0) {
      v.kr = 1.0;
      v.dkr = 0.0;
    } else {
      const double head = fabs(pc) / (P.density * P.gravity);
      v.kr = krt_lookup(P, head, 0);
      v.dkr = krt_lookup(P, head, 1);
    }
  }
  kr[c] = v.kr;
  dkr[c] = v.dkr;
  sat[c] = v.s;
  dsat[c] = v.ds;
}

__global__ void k_saturation(DevProblem P, const double *__restrict__ p, double *__restrict__ s) {
  pdl_enter();
  long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (c >= P.n) return;
  s[c] = vg_all(P, p[c], vg_at(P, c)).s;
}

// Residual (nl_function_eval.c:167-2323).  Accumulation order per cell
// follows the reference: accumulation, storage, sources, then the face
// fluxes scattered from the k-1, j-1, i-1 neighbours, the cell's own three
// upper faces, and finally the boundary patches in patch order.
// SURF: slopes and/or overland flow present (false: flat box, the lean path)
// VEL: also write the face velocities and overland fluxes (VelOut): interior
// faces as flux / area (nl_function_eval.c:845-848), boundary faces as the
// patch loops store them (vel_vec[vel_idx], :1227-1230, :1432, :1681-1687,
// :1775-1781), q_overlnd_x / y = ke, kn of the column (:1648-1656)
//
// residual_cell is everything of one cell's F but the interior face fluxes,
// which the caller supplies: the lower z / y / x faces (fl_z, fl_y, fl_x,
// used where k, j, i > 0) and the cell's own right / front / upper faces
// (0 on the domain's upper faces).  Both launch forms below pass the values
// of the same flux functions with the same operands, so their F is equal
// bit for bit.
template <bool SURF, bool VEL>
__device__ __forceinline__ void residual_cell(const DevProblem &P, int i, int j, int k,
                                              long long c, const double *__restrict__ p,
                                              const double *__restrict__ p_old,
                                              const double *__restrict__ s_old,
                                              const double *__restrict__ kr,
                                              const double *__restrict__ satv, double dt,
                                              double *__restrict__ f, const VelOut &V,
                                              double fl_z, double fl_y, double fl_x,
                                              double u_right, double u_front, double u_upper) {
  const long long sz = (long long)P.nx * P.ny;
  const double rho = P.density, g = P.gravity;
  const double vol = P.dx * P.dy * P.dz;
  const double zm = __ldg(P.zmult + k);
  const double pc = p[c];
  const double sat = satv[c];
  const double so = s_old[c];
  double fc = (sat * rho - so * rho) * P.porosity * vol * 1.0 * 1.0 * zm;
  fc += P.sstorage * vol * 1.0 * 1.0 * zm * (pc * sat * rho - p_old[c] * so * rho);
  fc -= vol * 1.0 * 1.0 * zm * dt * (0.0 + (P.et ? __ldg(P.et + c) : 0.0));
  const double kxc = __ldg(P.kx + c), kyc = __ldg(P.ky + c), kzc = __ldg(P.kz + c);
  const double krc = kr[c];
  // neighbours' scatter (reference loop order: plane k-1, row j-1, cell i-1)
  if (k > 0) fc += -dt * fl_z;
  if (j > 0) fc += -dt * fl_y;
  if (i > 0) fc += -dt * fl_x;
  fc += dt * (u_right + u_front + u_upper);
  if (VEL) {
    const long long fx1 = (long long)(P.nx + 1), cyz = (long long)P.nx * (P.ny + 1);
    if (V.vx && i + 1 < P.nx)
      V.vx[(i + 1) + fx1 * (j + (long long)P.ny * k)] = u_right / (P.dy * P.dz * zm * 1.0);
    if (V.vy && j + 1 < P.ny)
      V.vy[i + (long long)P.nx * (j + 1) + cyz * k] = u_front / (P.dx * P.dz * zm * 1.0);
    if (V.vz && k + 1 < P.nz) V.vz[c + sz] = u_upper / (P.dx * P.dy * 1.0 * 1.0);
  }

  // boundary patches (nl_function_eval.c:979-1435)
  const double ffx = P.dy * P.dz, ffy = P.dx * P.dz, ffz = P.dx * P.dy;
  const bool onf[6] = {i == 0, i == P.nx - 1, j == 0, j == P.ny - 1, k == 0, k == P.nz - 1};
#pragma unroll
  for (int face = 0; face < 6; face++) {
    if (!onf[face]) continue;
    const double value = __ldg(P.bc_val[face] + face_slot(P, face, i, j, k));
    const double dir = (face & 1) ? 1.0 : -1.0;
    double u_new;
    double vel = 0.0;  // this face's velocity (VEL)
    if (P.bc_type[face] == 0 || P.bc_type[face] == 5) {
      // FluxConst, or SeepageFace (nl_function_eval.c:1692-1784): a flux
      // face whose top face also drains the ponded water
      double q_ov = 0.0;
      if (P.bc_type[face] == 5 && face == 5) {
        q_ov = (vol / P.dz) * dt * (pmax0(pc) - 0.0);
        fc += q_ov;
      }
      double h = (face < 2) ? ffx * zm : (face < 4) ? ffy * zm : ffz;
      u_new = h * value;
      if (VEL) vel = (P.bc_type[face] == 0) ? value : (u_new + q_ov / dt) / h;
    } else if (SURF && P.bc_type[face] == 2) {
      // OverlandKinematic top face (nl_function_eval.c:1786-2000): ponding and
      // routing term, then the rain flux like FluxConst
      const OvCell o = ov_cell(P, i, j);
      double ke = -(o.sfx / (o.sq * o.n)) * pow(ov_press_x(P, p, i, j, o), (5.0 / 3.0));
      double kn = -(o.sfy / (o.sq * o.n)) * pow(ov_press_y(P, p, i, j, o), (5.0 / 3.0));
      double kw = 0.0, ks = 0.0;
      if (i > 0) {
        const OvCell ow = ov_cell(P, i - 1, j);
        kw = -(ow.sfx / (ow.sq * ow.n)) * pow(ov_press_x(P, p, i - 1, j, ow), (5.0 / 3.0));
      } else if (o.sfx > 0.0) {  // outflow through the lower x edge
        kw = -(o.sfx / (o.sq * o.n)) * pow(pmax0(pc), (5.0 / 3.0));
      }
      if (j > 0) {
        const OvCell os = ov_cell(P, i, j - 1);
        ks = -(os.sfy / (os.sq * os.n)) * pow(ov_press_y(P, p, i, j - 1, os), (5.0 / 3.0));
      } else if (o.sfy > 0.0) {  // outflow through the lower y edge
        ks = -(o.sfy / (o.sq * o.n)) * pow(pmax0(pc), (5.0 / 3.0));
      }
      const double q_ov = vol * (pmax0(pc) - pmax0(p_old[c])) / P.dz +
                          dt * vol * ((ke - kw) / P.dx + (kn - ks) / P.dy) / P.dz;
      fc += q_ov;
      u_new = ffz * value;
      if (VEL) {
        vel = (u_new + q_ov / dt) / ffz;
        if (V.qx) V.qx[i + (long long)P.nx * j] = ke;
        if (V.qy) V.qy[i + (long long)P.nx * j] = kn;
      }
    } else if (SURF && P.bc_type[face] == 4) {
      // OverlandFlow top face (nl_function_eval.c:1437-1690): each face flux
      // is the upwind part of the two columns' own fluxes, plus the spin-up
      // damping term; with OverlandFlowSpinUp the ponded head drains in
      // place of the ponding and routing term (:1659-1673)
      const double qw = ovf_q<true>(P, p, i - 1, j), qc = ovf_q<true>(P, p, i, j),
                   qe = ovf_q<true>(P, p, i + 1, j);
      const double kw = pmax0(qw) - pmax0(-qc), ke = pmax0(qc) - pmax0(-qe);
      const double qs = ovf_q<false>(P, p, i, j - 1), qm = ovf_q<false>(P, p, i, j),
                   qn = ovf_q<false>(P, p, i, j + 1);
      const double ks = pmax0(qs) - pmax0(-qm), kn = pmax0(qm) - pmax0(-qn);
      double q_ov = vol * (pmax0(pc) - pmax0(p_old[c])) / P.dz +
                    dt * vol * ((ke - kw) / P.dx + (kn - ks) / P.dy) / P.dz;
      if (P.ov_p2 != 0.0 || P.ov_spinup == 1) {
        const double damp = exp(fmin(pc, 0.0) * P.ov_p1) * P.ov_p2;
        q_ov = q_ov + vol * dt / P.dz * damp;
        if (P.ov_spinup == 1) q_ov = (vol / P.dz) * dt * ((pmax0(pc) - 0.0) + damp);
      }
      fc += q_ov;
      u_new = ffz * value;
      if (VEL) {
        vel = (u_new + q_ov / dt) / ffz;
        if (V.qx) V.qx[i + (long long)P.nx * j] = ke;
        if (V.qy) V.qy[i + (long long)P.nx * j] = kn;
      }
    } else if (SURF && P.bc_type[face] == 3) {
      // OverlandDiffusive top face (nl_function_eval.c:2028-2259): the same
      // ponding and routing term with the diffusive-wave face fluxes
      const OvdCol o = ovd_col(P, p, i, j);
      double qxw, qys;
      ovd_q_edges(P, o, i, j, qxw, qys);
      const double ke = ovd_qx(o), kn = ovd_qy(o);
      const double kw = i > 0 ? ovd_qx(ovd_col(P, p, i - 1, j)) : qxw;
      const double ks = j > 0 ? ovd_qy(ovd_col(P, p, i, j - 1)) : qys;
      const double q_ov = vol * (pmax0(pc) - pmax0(p_old[c])) / P.dz +
                          dt * vol * ((ke - kw) / P.dx + (kn - ks) / P.dy) / P.dz;
      fc += q_ov;
      u_new = ffz * value;
      if (VEL) {
        vel = (u_new + q_ov / dt) / ffz;
        if (V.qx) V.qx[i + (long long)P.nx * j] = ke;
        if (V.qy) V.qy[i + (long long)P.nx * j] = kn;
      }
    } else {
      const VG v = vg_at(P, c);
      double krg = vg_kr(P, value, v.alpha, v.n);
      if (face < 4) {
        double h = (face < 2) ? ffx * zm : ffy * zm;
        double kk = (face < 2) ? kxc : kyc;
        double dd = (face < 2) ? P.dx : P.dy;
        if (dir < 0) {
          double diff = value - pc;
          u_new = upstream(value, pc, krg * rho, krc * rho);
          u_new = u_new * h * (kk * P.inv_visc) * 2.0 * (diff / dd);
        } else {
          double diff = pc - value;
          u_new = upstream(pc, value, krc * rho, krg * rho);
          u_new = u_new * h * (kk * P.inv_visc) * 2.0 * (diff / dd);
        }
      } else {
        double sep = P.dz * zm;
        double lower, upper;
        if (dir < 0) {
          lower = value / sep - 0.25 * rho * g;
          upper = pc / sep + 0.25 * rho * g;
          u_new = upstream(lower, upper, krg * rho, krc * rho);
        } else {
          lower = (pc / sep) - 0.25 * rho * g * 1.0;
          upper = (value / sep) + 0.25 * rho * g * 1.0;
          u_new = upstream(lower, upper, krc * rho, krg * rho);
        }
        u_new = u_new * ffz * (kzc * P.inv_visc) * 2.0 * (lower - upper);
      }
      // DirichletBC: u_new / h (nl_function_eval.c:1227-1230)
      if (VEL) vel = u_new / ((face < 2) ? ffx * zm : (face < 4) ? ffy * zm : ffz);
    }
    fc += dt * dir * u_new;
    if (VEL) {
      const int up = face & 1;
      if (face < 2 && V.vx)
        V.vx[(i + up) + (long long)(P.nx + 1) * (j + (long long)P.ny * k)] = vel;
      else if (face >= 2 && face < 4 && V.vy)
        V.vy[i + (long long)P.nx * (j + up) + (long long)P.nx * (P.ny + 1) * k] = vel;
      else if (face >= 4 && V.vz)
        V.vz[c + up * sz] = vel;
    }
  }
  f[c] = fc;
}

// Gather form: every cell evaluates all six of its face fluxes (a face shared
// by two cells is evaluated by both, with the same operands in the same
// order).  The default launch form.
template <bool SURF, bool VEL = false>
__global__ void __launch_bounds__(256, 5) k_residual(DevProblem P, const double *__restrict__ p,
                           const double *__restrict__ p_old, const double *__restrict__ s_old,
                           const double *__restrict__ kr, const double *__restrict__ satv,
                           double dt, double *__restrict__ f, VelOut V = VelOut{}) {
  pdl_enter();
  if (P.dtp) dt = *P.dtp;
  int i, j, k;
  if (!launch_ijk(P.nx, P.ny, P.nz, i, j, k)) return;
  const long long c = i + (long long)P.nx * (j + (long long)P.ny * k);
  const long long sy = P.nx, sz = (long long)P.nx * P.ny;
  const double g = P.gravity;
  const double zm = __ldg(P.zmult + k);
  const double pc = p[c];
  const double kxc = __ldg(P.kx + c), kyc = __ldg(P.ky + c), kzc = __ldg(P.kz + c);
  const double krc = kr[c];
  double fl_z = 0.0, fl_y = 0.0, fl_x = 0.0;
  if (k > 0) {
    long long l = c - sz;
    double zl = __ldg(P.zmult + k - 1);
    fl_z = flux_z(P, p[l], pc, __ldg(P.kz + l), kzc, kr[l], krc, zl, zm, k - 1);
    if (P.fbz) fl_z = fl_z * fb_z(P, l);
  }
  double gs = 0.5 * (g * 0.0 + g * 0.0), gc = 0.5 * (g * 1.0 + g * 1.0);
  if (j > 0) {
    long long s = c - sy;
    if (SURF) tfg_face_y(P, i, j - 1, gs, gc);
    fl_y = flux_y(P, p[s], pc, __ldg(P.ky + s), kyc, kr[s], krc, zm, gs, gc);
    if (P.fby) fl_y = fl_y * fb_y(P, s);
  }
  if (i > 0) {
    long long w = c - 1;
    if (SURF) tfg_face_x(P, i - 1, j, gs, gc);
    fl_x = flux_x(P, p[w], pc, __ldg(P.kx + w), kxc, kr[w], krc, zm, gs, gc);
    if (P.fbx) fl_x = fl_x * fb_x(P, w);
  }
  double u_right = 0.0, u_front = 0.0, u_upper = 0.0;
  if (i + 1 < P.nx) {
    long long e = c + 1;
    if (SURF) tfg_face_x(P, i, j, gs, gc);
    u_right = flux_x(P, pc, p[e], kxc, __ldg(P.kx + e), krc, kr[e], zm, gs, gc);
    if (P.fbx) u_right = u_right * fb_x(P, c);
  }
  if (j + 1 < P.ny) {
    long long nn = c + sy;
    if (SURF) tfg_face_y(P, i, j, gs, gc);
    u_front = flux_y(P, pc, p[nn], kyc, __ldg(P.ky + nn), krc, kr[nn], zm, gs, gc);
    if (P.fby) u_front = u_front * fb_y(P, c);
  }
  if (k + 1 < P.nz) {
    long long u = c + sz;
    u_upper = flux_z(P, pc, p[u], kzc, __ldg(P.kz + u), krc, kr[u], zm,
                     __ldg(P.zmult + k + 1), k);
    if (P.fbz) u_upper = u_upper * fb_z(P, c);
  }
  residual_cell<SURF, VEL>(P, i, j, k, c, p, p_old, s_old, kr, satv, dt, f, V, fl_z, fl_y, fl_x,
                           u_right, u_front, u_upper);
}

// Face-once form: a block owns a (blockDim.x x blockDim.y) column tile of
// planes k0 .. k0+kchunk-1 and walks up through them.  Each cell evaluates
// only its right, front and upper faces; the right / front fluxes go to shared
// memory for the neighbour in the tile, the upper flux stays in a register as
// the lower flux of the next plane.  The tile's west / south edge faces and
// the chunk's first lower faces are evaluated by the cells on those edges.
// Every flux is the same function of the same operands as in the gather form.
// Shared memory: blockDim.y x (blockDim.x + 1) right fluxes and
// (blockDim.y + 1) x blockDim.x front fluxes.
template <bool SURF, bool VEL = false>
__global__ void __launch_bounds__(256) k_residual_zm(DevProblem P, const double *__restrict__ p,
                           const double *__restrict__ p_old, const double *__restrict__ s_old,
                           const double *__restrict__ kr, const double *__restrict__ satv,
                           double dt, double *__restrict__ f, VelOut V, int kchunk) {
  extern __shared__ double zm_smem[];
  const int bx = blockDim.x, by = blockDim.y, tx = threadIdx.x, ty = threadIdx.y;
  double *sE = zm_smem;                    // [by][bx + 1]: sE[ty][tx + 1] = right face of (tx, ty)
  double *sN = zm_smem + by * (bx + 1);    // [by + 1][bx]: sN[ty + 1][tx] = front face
  pdl_enter();
  if (P.dtp) dt = *P.dtp;
  const int i = blockIdx.x * bx + tx, j = blockIdx.y * by + ty;
  const int k0 = blockIdx.z * kchunk, k1 = min(P.nz, k0 + kchunk);
  const bool in = i < P.nx && j < P.ny;
  const long long sy = P.nx, sz = (long long)P.nx * P.ny;
  const double g = P.gravity;
  // gravity terms of this column's faces (constant through the planes)
  double gsw = 0.5 * (g * 0.0 + g * 0.0), gcw = 0.5 * (g * 1.0 + g * 1.0);
  double gss = gsw, gcs = gcw, gse = gsw, gce = gcw, gsn = gsw, gcn = gcw;
  if (SURF && in) {
    if (i > 0) tfg_face_x(P, i - 1, j, gsw, gcw);
    if (j > 0) tfg_face_y(P, i, j - 1, gss, gcs);
    if (i + 1 < P.nx) tfg_face_x(P, i, j, gse, gce);
    if (j + 1 < P.ny) tfg_face_y(P, i, j, gsn, gcn);
  }
  long long c = i + (long long)P.nx * (j + (long long)P.ny * k0);
  double fl_z = 0.0;
  if (in && k0 > 0 && k0 < k1)
    fl_z = flux_z(P, p[c - sz], p[c], __ldg(P.kz + c - sz), __ldg(P.kz + c), kr[c - sz], kr[c],
                  __ldg(P.zmult + k0 - 1), __ldg(P.zmult + k0), k0 - 1) *
           fb_z(P, c - sz);
  for (int k = k0; k < k1; k++, c += sz) {
    double u_right = 0.0, u_front = 0.0, u_upper = 0.0;
    if (in) {
      const double zm = __ldg(P.zmult + k);
      const double pc = p[c];
      const double kxc = __ldg(P.kx + c), kyc = __ldg(P.ky + c), kzc = __ldg(P.kz + c);
      const double krc = kr[c];
      if (i + 1 < P.nx)
        u_right = flux_x(P, pc, p[c + 1], kxc, __ldg(P.kx + c + 1), krc, kr[c + 1], zm, gse,
                         gce) *
                  fb_x(P, c);
      if (j + 1 < P.ny)
        u_front = flux_y(P, pc, p[c + sy], kyc, __ldg(P.ky + c + sy), krc, kr[c + sy], zm, gsn,
                         gcn) *
                  fb_y(P, c);
      if (k + 1 < P.nz)
        u_upper = flux_z(P, pc, p[c + sz], kzc, __ldg(P.kz + c + sz), krc, kr[c + sz], zm,
                         __ldg(P.zmult + k + 1), k) *
                  fb_z(P, c);
      // the tile's west and south edge faces
      if (tx == 0 && i > 0)
        sE[ty * (bx + 1)] = flux_x(P, p[c - 1], pc, __ldg(P.kx + c - 1), kxc, kr[c - 1], krc, zm,
                                   gsw, gcw) *
                            fb_x(P, c - 1);
      if (ty == 0 && j > 0)
        sN[tx] = flux_y(P, p[c - sy], pc, __ldg(P.ky + c - sy), kyc, kr[c - sy], krc, zm, gss,
                        gcs) *
                 fb_y(P, c - sy);
    }
    sE[ty * (bx + 1) + tx + 1] = u_right;
    sN[(ty + 1) * bx + tx] = u_front;
    __syncthreads();
    if (in)
      residual_cell<SURF, VEL>(P, i, j, k, c, p, p_old, s_old, kr, satv, dt, f, V, fl_z,
                               sN[ty * bx + tx], sE[ty * (bx + 1) + tx], u_right, u_front,
                               u_upper);
    fl_z = u_upper;
    __syncthreads();
  }
}

// Flux derivatives of one x (or y) face between a (left) and b (right)
// (richards_jacobian_eval.c:618-660): returns west/east and symmetric parts.
// TA is the arithmetic of the face terms: double for the FP64 Jacobian; for
// a Jacobian stored in FP32 the face terms are formed in FP32 too (their
// products round no worse than the storage), while the upwind decisions, the
// pressure differences they come from and the row sums stay FP64.  With TA =
// double the operations are those of the reference macros, in their order.
template <typename TA>
struct FaceDer {
  TA lo, hi, sym;  // d/dp of the face flux w.r.t. lower cell (negated), upper cell; sym part
};

template <typename TA>
__device__ __forceinline__ TA harmonic_t(TA a, TA b) {
  return (a + b) ? (TA(2) * a * b) / (a + b) : TA(0);
}
template <typename TA>
__device__ __forceinline__ TA harmonic_dz_t(TA a, TA b, TA c, TA d) {
  return ((c * b) + (a * d)) ? (((c + d) * a * b) / ((b * c) + (a * d))) : TA(0);
}
// upstream() with the decision taken in FP64 and the values in TA
template <typename TA>
__device__ __forceinline__ TA pick(double a, double b, TA c, TA d) {
  return ((a - b) >= 0) ? c : d;
}

template <typename TA>
__device__ __forceinline__ FaceDer<TA> face_der_xy(const DevProblem &P, double dt, double fb,
                                                   double h_ff,
                                                   double dd, double inv_dd, double pa,
                                                   double pb, double ka, double kb, double prod,
                                                   double prod_der, double prod_rt,
                                                   double prod_rt_der, double zm, double dir_g,
                                                   double dir_g_c) {
  const double diff64 = pa - pb;
  const double updir = (diff64 * inv_dd) * dir_g_c - dir_g;
  const TA diff = (TA)diff64;
  // x_coeff / y_coeff (richards_jacobian_eval.c:662, 692): FB * dt * ...
  const TA coeff = (TA)fb * (TA)dt * (TA)h_ff * (TA)inv_dd * (TA)zm *
                   harmonic_t<TA>((TA)ka, (TA)kb) * (TA)P.inv_visc;
  const TA dgc = (TA)dir_g_c, dg = (TA)dir_g, tdd = (TA)dd;
  FaceDer<TA> r;
  TA sym_lo = (-coeff * pick<TA>(updir, 0.0, (TA)prod, (TA)prod_rt)) * dgc;
  r.lo = (-coeff * diff * pick<TA>(updir, 0.0, (TA)prod_der, TA(0.0))) * dgc + sym_lo;
  r.lo += (coeff * tdd * pick<TA>(updir, 0.0, (TA)prod_der, TA(0.0))) * dg;
  r.sym = (-coeff * pick<TA>(updir, 0.0, (TA)prod, (TA)prod_rt)) * dgc;
  r.hi = (coeff * diff * pick<TA>(updir, 0.0, TA(0.0), (TA)prod_rt_der)) * dgc + r.sym;
  r.hi += -(coeff * tdd * pick<TA>(updir, 0.0, TA(0.0), (TA)prod_rt_der)) * dg;
  return r;
}

// z face between a (lower) and b (upper) (richards_jacobian_eval.c:697-745)
template <typename TA>
__device__ __forceinline__ FaceDer<TA> face_der_z(const DevProblem &P, double dt, double fb,
                                                  double pa,
                                                  double pb, double ka, double kb, double prod,
                                                  double prod_der, double prod_up,
                                                  double prod_up_der, double za, double zb,
                                                  int k) {
  const double g = P.gravity, rho = P.density, drho = 0.0;
  const double dz = P.dz;
  const double inv_sep = __ldg(P.zface + 3 * k);
  double lower_cond = pa * inv_sep - __ldg(P.zface + 3 * k + 1) * rho * g;
  double upper_cond = pb * inv_sep + __ldg(P.zface + 3 * k + 2) * rho * g;
  const TA diff = (TA)(lower_cond - upper_cond);
  const TA z_coeff = (TA)fb * (TA)dt * ((TA)P.dx * (TA)P.dy) *
                     harmonic_dz_t<TA>((TA)ka, (TA)kb, (TA)za, (TA)zb) * (TA)P.inv_visc;
  const TA up = pick<TA>(lower_cond, upper_cond, (TA)prod, (TA)prod_up);
  const TA grav = (TA)(-g * 0.5 * dz * (amean(za, zb)) * drho);
  const TA sym_lower = -z_coeff * (TA)inv_sep * up;
  FaceDer<TA> r;
  r.lo = -z_coeff * (diff * pick<TA>(lower_cond, upper_cond, (TA)prod_der, TA(0.0)) +
                     (grav * up)) +
         sym_lower;
  r.sym = z_coeff * (TA)inv_sep * -up;
  r.hi = z_coeff * (diff * pick<TA>(lower_cond, upper_cond, TA(0.0), (TA)prod_up_der) +
                    (grav * up)) +
         r.sym;
  return r;
}

// Jacobian assembly (richards_jacobian_eval.c:217-1420).  Writes the full
// 7-point J (C W E S N L U, FP64 or FP32) and the symmetric preconditioner
// matrix (C E N U: full diagonal, symmetric off-diagonal parts; PCMatrixType
// PFSymmetric), in the preconditioner's precision.
//
// jacobian_cell is everything of one cell's row but the interior face
// derivatives, which the caller supplies: the lower z / y / x faces' (lo, hi)
// parts (used where k, j, i > 0) and the cell's own upper faces (zero on the
// domain's upper faces).  Both launch forms below pass the values of the
// same face functions with the same operands, so their J and PC matrix are
// equal bit for bit.
template <typename TA>
struct FaceLH {
  TA lo, hi;
};

template <typename TJ, typename TP, bool SURF>
__device__ __forceinline__ void jacobian_cell(const DevProblem &P, int i, int j, int k,
                                              long long c, const double *__restrict__ p,
                                              const double *__restrict__ kr,
                                              const double *__restrict__ dkr,
                                              const double *__restrict__ satv,
                                              const double *__restrict__ dsatv, double dt,
                                              const JacOut<TJ> &J, const PCOut<TP> &M,
                                              FaceLH<TJ> dl_z, FaceLH<TJ> dl_y, FaceLH<TJ> dl_x,
                                              const FaceDer<TJ> &de, const FaceDer<TJ> &dn,
                                              const FaceDer<TJ> &du) {
  const long long sy = P.nx;
  const double rho = P.density, g = P.gravity, drho = 0.0;
  const double vol = P.dx * P.dy * P.dz;
  const double ffx = P.dy * P.dz, ffy = P.dx * P.dz, ffz = P.dx * P.dy;
  const double zm = __ldg(P.zmult + k);
  const double pc = p[c];
  const double sat = satv[c], dsat = dsatv[c];
  const double prod = kr[c] * rho, prod_der = dkr[c] * rho + kr[c] * drho;
  const double kxc = __ldg(P.kx + c), kyc = __ldg(P.ky + c), kzc = __ldg(P.kz + c);
  (void)g;
  (void)kzc;

  double vol2 = vol * zm;
  double cp = 0.0;
  cp += (dsat * rho + sat * drho) * P.porosity * vol2 +
        P.sstorage * vol2 * (dsat * rho * pc + sat * drho * pc + sat * rho);

  double w = 0.0, s = 0.0, l = 0.0, e = 0.0, nn = 0.0, u = 0.0;
  double es = 0.0, ns = 0.0, us = 0.0;
  if (k > 0) {
    cp += -dl_z.hi;
    l = dl_z.lo;
  }
  if (j > 0) {
    cp += -dl_y.hi;
    s = dl_y.lo;
  }
  if (i > 0) {
    cp += -dl_x.hi;
    w = dl_x.lo;
  }
  double west_t = 0.0, south_t = 0.0, lower_t = 0.0;
  if (i + 1 < P.nx) {
    west_t = de.lo;
    e = de.hi;
    es = de.sym;
  }
  if (j + 1 < P.ny) {
    south_t = dn.lo;
    nn = dn.hi;
    ns = dn.sym;
  }
  if (k + 1 < P.nz) {
    lower_t = du.lo;
    u = du.hi;
    us = du.sym;
  }
  cp += -(west_t + south_t + lower_t);

  // Dirichlet patches (richards_jacobian_eval.c:1049-1200); flux patches
  // leave the row as is (their boundary entries are zero)
  const bool onf[6] = {i == 0, i == P.nx - 1, j == 0, j == P.ny - 1, k == 0, k == P.nz - 1};
#pragma unroll
  for (int face = 0; face < 6; face++) {
    if (!onf[face] || P.bc_type[face] != 1) continue;
    const double value = __ldg(P.bc_val[face] + face_slot(P, face, i, j, k));
    const double den_d = rho;
    const VG v = vg_at(P, c);
    const double prod_val = vg_kr(P, value, v.alpha, v.n) * den_d;
    // above the top layer the z_mult ghost keeps the 1 it was initialised
    // with (problem_dz_scale.c:92)
    const double zu = (k + 1 < P.nz) ? __ldg(P.zmult + k + 1) : 1.0;
    double coeff, diff, o_temp;
    switch (face) {
      case 0:
        coeff = dt * ffx * zm * (2.0 / P.dx) * kxc * P.inv_visc;
        diff = value - pc;
        o_temp = coeff * (diff * upstream(value, pc, 0.0, prod_der) -
                          upstream(value, pc, prod_val, prod));
        break;
      case 1:
        coeff = dt * ffx * zm * (2.0 / P.dx) * kxc * P.inv_visc;
        diff = pc - value;
        o_temp = -coeff * (diff * upstream(pc, value, prod_der, 0.0) +
                           upstream(pc, value, prod, prod_val));
        break;
      case 2:
        coeff = dt * ffy * zm * (2.0 / P.dy) * kyc * P.inv_visc;
        diff = value - pc;
        o_temp = coeff * (diff * upstream(value, pc, 0.0, prod_der) -
                          upstream(value, pc, prod_val, prod));
        break;
      case 3:
        coeff = dt * ffy * zm * (2.0 / P.dy) * kyc * P.inv_visc;
        diff = pc - value;
        o_temp = -coeff * (diff * upstream(pc, value, prod_der, 0.0) +
                           upstream(pc, value, prod, prod_val));
        break;
      case 4: {
        coeff = dt * ffz * (2.0 / (P.dz * amean(zm, zu))) * kzc * P.inv_visc;
        double lc = (value)-0.5 * P.dz * zm * den_d * g;
        double uc = (pc) + 0.5 * P.dz * zm * rho * g;
        diff = lc - uc;
        o_temp = coeff * (diff * upstream(lc, uc, 0.0, prod_der) +
                          ((-1.0 - g * 0.5 * P.dz * zm * drho) * upstream(lc, uc, prod_val, prod)));
        break;
      }
      default: {
        coeff = dt * ffz * (2.0 / (P.dz * amean(zm, zu))) * kzc * P.inv_visc;
        double lc = (pc)-0.5 * P.dz * zm * rho * g;
        double uc = (value) + 0.5 * P.dz * zm * den_d * g;
        diff = lc - uc;
        o_temp = -coeff * (diff * upstream(lc, uc, prod_der, 0.0) +
                           ((1.0 - g * 0.5 * P.dz * zm * drho) * upstream(lc, uc, prod, prod_val)));
        break;
      }
    }
    cp -= o_temp;
  }

  // SeepageFace on the top face (richards_jacobian_eval.c:1319-1345), in
  // patch order after the Dirichlet corrections
  if (k == P.nz - 1 && P.bc_type[5] == 5 && pc >= 0.0) cp += (vol / P.dz) * dt * (1.0 + 0.0);

  // kinematic overland terms of a top cell, MGSemi form
  // (richards_jacobian_eval.c:1863-1990, CALCDER of overlandflow_eval_Kin.c),
  // added after every other term.  In the symmetric storage the west / south
  // terms belong to the neighbour's E / N entry (lower coefficient aliasing,
  // matrix.c:484-490): E(i) gets this cell's east term, then the east
  // neighbour's west term, in the reference's loop order.
  // difference-quotient mode: an OverlandFlow top cell with p > 0 gets
  // vol zm / (dz mean(zm, 1)) (dt + 1), the z_mult ghost above the top layer
  // keeping its initial 1 (problem_dz_scale.c:92), and no surface terms
  if (M.fd && k == P.nz - 1 && P.bc_type[5] == 4 && pc > 0.0)
    cp += (vol * zm) / (P.dz * (0.5 * (zm + 1.0))) * (dt + 1);
  if (SURF && !M.fd && k == P.nz - 1 && P.bc_type[5] == 2) {
    const double cx = (vol / ffy) * dt, cy = (vol / ffx) * dt;
    const double two3 = 2.0 / 3.0;
    const OvCell o = ov_cell(P, i, j);
    const double qxt = -(5.0 / 3.0) * (o.sfx / (o.sq * o.n)) * pow(ov_press_x(P, p, i, j, o), two3);
    const double qyt = -(5.0 / 3.0) * (o.sfy / (o.sq * o.n)) * pow(ov_press_y(P, p, i, j, o), two3);
    const double ke_d = pmax0(qxt), kn_d = pmax0(qyt);
    double kw_d = 0.0, ks_d = 0.0, ke_w = 0.0, kn_s = 0.0;
    if (i > 0) {
      const OvCell ow = ov_cell(P, i - 1, j);
      const double q = -(5.0 / 3.0) * (ow.sfx / (ow.sq * ow.n)) *
                       pow(ov_press_x(P, p, i - 1, j, ow), two3);
      kw_d = -pmax0(-q);
      ke_w = pmax0(q);
    } else if (o.sfx > 0.0) {
      const double q = -(5.0 / 3.0) * (o.sfx / (o.sq * o.n)) * pow(pmax0(pc), two3);
      kw_d = -pmax0(-q);
      ke_w = pmax0(q);
    }
    if (j > 0) {
      const OvCell os = ov_cell(P, i, j - 1);
      const double q = -(5.0 / 3.0) * (os.sfy / (os.sq * os.n)) *
                       pow(ov_press_y(P, p, i, j - 1, os), two3);
      ks_d = -pmax0(-q);
      kn_s = pmax0(q);
    } else if (o.sfy > 0.0) {
      const double q = -(5.0 / 3.0) * (o.sfy / (o.sq * o.n)) * pow(pmax0(pc), two3);
      ks_d = -pmax0(-q);
      kn_s = pmax0(q);
    }
    if (pc > 0.0)
      cp += (vol / P.dz) + cx * (ke_d - kw_d) + cy * (kn_d - ks_d);
    const double tw = cx * (ke_w), te = cx * (-pmax0(-qxt));
    const double ts = cy * (kn_s), tn = cy * (-pmax0(-qyt));
    w -= tw;
    e += te;
    s -= ts;
    nn += tn;
    es += te;
    if (i + 1 < P.nx) es -= cx * (ke_d);  // the east neighbour's west term
    ns += tn;
    if (j + 1 < P.ny) ns -= cy * (kn_d);  // the north neighbour's south term
  }
  // OverlandFlow terms of a top cell, MGSemi form
  // (richards_jacobian_eval.c:2028-2090, CALCDER of overlandflow_eval.c):
  // the derivative parts of each column's own flux; neighbours' parts give
  // the off-diagonals, and the east neighbour's west term lands in E(i)
  // With OverlandFlowSpinUp the patch's own diagonal term of a cell with
  // p >= 0 comes first (richards_jacobian_eval.c:1258-1268) and the
  // derivative parts are zero (their evaluation is skipped, :1287); a
  // non-ponded cell gets the derivative of the spin-up damping term.
  if (SURF && !M.fd && k == P.nz - 1 && P.bc_type[5] == 4) {
    const bool spin = P.ov_spinup == 1;
    if (spin && pc >= 0.0) cp += (vol / P.dz) * dt * (1.0 + 0.0);
    const double cx = (vol / ffy) * dt, cy = (vol / ffx) * dt;
    const double qx = spin ? 0.0 : ovf_qder<true>(P, pc, i, j);
    const double qy = spin ? 0.0 : ovf_qder<false>(P, pc, i, j);
    const double ke_d = pmax0(qx), kw_d = -pmax0(-qx);
    const double kn_d = pmax0(qy), ks_d = -pmax0(-qy);
    // the neighbours' derivative parts: ke of i-1, kw of i+1, kn of j-1, ks of j+1
    const double ke_w = i > 0 && !spin ? pmax0(ovf_qder<true>(P, p[c - 1], i - 1, j)) : 0.0;
    const double kw_e =
        i + 1 < P.nx && !spin ? -pmax0(-ovf_qder<true>(P, p[c + 1], i + 1, j)) : 0.0;
    const double kn_s = j > 0 && !spin ? pmax0(ovf_qder<false>(P, p[c - sy], i, j - 1)) : 0.0;
    const double ks_n =
        j + 1 < P.ny && !spin ? -pmax0(-ovf_qder<false>(P, p[c + sy], i, j + 1)) : 0.0;
    if (pc > 0.0)
      cp += (vol / P.dz) + cx * (ke_d - kw_d) + cy * (kn_d - ks_d);
    else
      cp += 0.0 + dt * (vol / P.dz) * (P.ov_p1 * exp(fmin(pc, 0.0) * P.ov_p1) * P.ov_p2);
    const double tw = cx * (ke_w), te = cx * (kw_e);
    const double ts = cy * (kn_s), tn = cy * (ks_n);
    w -= tw;
    e += te;
    s -= ts;
    nn += tn;
    es += te;
    if (i + 1 < P.nx) es -= cx * (ke_d);  // the east neighbour's west term
    ns += tn;
    if (j + 1 < P.ny) ns -= cy * (kn_d);  // the north neighbour's south term
  }
  // diffusive overland terms of a top cell, MGSemi form
  // (richards_jacobian_eval.c:1989-2026, CALCDER of
  // overlandflow_eval_diffusive.c): off-diagonals from the non-symmetric
  // derivative parts.  In the symmetric storage the west term of an i = 0
  // cell lands in the x_lower ghost column of E, which MGSemi's setup reads:
  // it is returned in wgv for the multigrid's ghost plane.
  double wgv = 0.0;
  if (SURF && !M.fd && k == P.nz - 1 && P.bc_type[5] == 3) {
    const double cx = (vol / ffy) * dt, cy = (vol / ffx) * dt;
    const OvdCol o = ovd_col(P, p, i, j);
    double ke_d, kens, kn_d, knns;
    ovd_der_x(P, o, ke_d, kens);
    ovd_der_y(P, o, kn_d, knns);
    double kw_d = 0.0, kwns = 0.0, ks_d = 0.0, ksns = 0.0;
    ovd_der_edges(P, o, i, j, kw_d, kwns, ks_d, ksns);
    if (i > 0) ovd_der_x(P, ovd_col(P, p, i - 1, j), kwns, kw_d);
    if (j > 0) ovd_der_y(P, ovd_col(P, p, i, j - 1), ksns, ks_d);
    if (pc > 0.0)
      cp += (vol / P.dz) + cx * (ke_d - kw_d) + cy * (kn_d - ks_d);
    const double tw = cx * (kwns), te = cx * (kens);
    const double ts = cy * (ksns), tn = cy * (knns);
    w -= tw;
    e += te;
    s -= ts;
    nn += tn;
    if (i == 0) wgv -= tw;
    es += te;
    if (i + 1 < P.nx) es -= cx * (ke_d);  // the east neighbour's west term
    ns += tn;
    if (j + 1 < P.ny) ns -= cy * (kn_d);  // the north neighbour's south term
  }
  if (J.c) {
    J.c[c] = (TJ)cp;
    J.w[c] = (TJ)w;
    J.e[c] = (TJ)e;
    J.s[c] = (TJ)s;
    J.n[c] = (TJ)nn;
    J.l[c] = (TJ)l;
    J.u[c] = (TJ)u;
  }
  if (M.c) {
    M.c[c] = (TP)cp;
    M.e[c] = (TP)es;
    M.n[c] = (TP)ns;
    M.u[c] = (TP)us;
    if (M.wg && i == 0) M.wg[j + (long long)P.ny * k] = (TP)wgv;
  }
}

// Gather form: every cell evaluates the derivative parts of all six of its
// faces.  The default launch form (see residual_gather).
template <typename TJ, typename TP, bool SURF>
__global__ void __launch_bounds__(128, 8) k_jacobian(DevProblem P, const double *__restrict__ p,
                           const double *__restrict__ kr, const double *__restrict__ dkr,
                           const double *__restrict__ satv, const double *__restrict__ dsatv,
                           double dt, JacOut<TJ> J, PCOut<TP> M) {
  pdl_enter();
  if (P.dtp) dt = *P.dtp;
  using TA = TJ;  // arithmetic of the face terms (see face_der_xy)
  int i, j, k;
  if (!launch_ijk(P.nx, P.ny, P.nz, i, j, k)) return;
  const long long c = i + (long long)P.nx * (j + (long long)P.ny * k);
  const long long sy = P.nx, sz = (long long)P.nx * P.ny;
  const double rho = P.density, g = P.gravity, drho = 0.0;
  const double ffx = P.dy * P.dz, ffy = P.dx * P.dz;
  const double zm = __ldg(P.zmult + k);
  const double pc = p[c];
  const double prod = kr[c] * rho, prod_der = dkr[c] * rho + kr[c] * drho;
  const double kxc = __ldg(P.kx + c), kyc = __ldg(P.ky + c), kzc = __ldg(P.kz + c);
  FaceLH<TA> dl_z{}, dl_y{}, dl_x{};
  FaceDer<TA> de{}, dn{}, du{};
  if (k > 0) {
    long long q = c - sz;
    FaceDer<TA> d = face_der_z<TA>(P, dt, fb_z(P, q), p[q], pc, __ldg(P.kz + q), kzc,
                                   kr[q] * rho, dkr[q] * rho + kr[q] * drho, prod, prod_der,
                                   __ldg(P.zmult + k - 1), zm, k - 1);
    dl_z = {d.lo, d.hi};
  }
  double gs = 0.5 * (g * 0.0 + g * 0.0), gc = 0.5 * (g * 1.0 + g * 1.0);
  if (j > 0) {
    long long q = c - sy;
    if (SURF) tfg_face_y(P, i, j - 1, gs, gc);
    FaceDer<TA> d = face_der_xy<TA>(P, dt, fb_y(P, q), ffy, P.dy, P.inv_dy, p[q], pc,
                                    __ldg(P.ky + q), kyc, kr[q] * rho,
                                    dkr[q] * rho + kr[q] * drho, prod, prod_der, zm, gs, gc);
    dl_y = {d.lo, d.hi};
  }
  if (i > 0) {
    long long q = c - 1;
    if (SURF) tfg_face_x(P, i - 1, j, gs, gc);
    FaceDer<TA> d = face_der_xy<TA>(P, dt, fb_x(P, q), ffx, P.dx, P.inv_dx, p[q], pc,
                                    __ldg(P.kx + q), kxc, kr[q] * rho,
                                    dkr[q] * rho + kr[q] * drho, prod, prod_der, zm, gs, gc);
    dl_x = {d.lo, d.hi};
  }
  if (i + 1 < P.nx) {
    long long q = c + 1;
    if (SURF) tfg_face_x(P, i, j, gs, gc);
    de = face_der_xy<TA>(P, dt, fb_x(P, c), ffx, P.dx, P.inv_dx, pc, p[q], kxc, __ldg(P.kx + q),
                         prod, prod_der, kr[q] * rho, dkr[q] * rho + kr[q] * drho, zm, gs, gc);
  }
  if (j + 1 < P.ny) {
    long long q = c + sy;
    if (SURF) tfg_face_y(P, i, j, gs, gc);
    dn = face_der_xy<TA>(P, dt, fb_y(P, c), ffy, P.dy, P.inv_dy, pc, p[q], kyc, __ldg(P.ky + q),
                         prod, prod_der, kr[q] * rho, dkr[q] * rho + kr[q] * drho, zm, gs, gc);
  }
  if (k + 1 < P.nz) {
    long long q = c + sz;
    du = face_der_z<TA>(P, dt, fb_z(P, c), pc, p[q], kzc, __ldg(P.kz + q), prod, prod_der,
                        kr[q] * rho, dkr[q] * rho + kr[q] * drho, zm, __ldg(P.zmult + k + 1), k);
  }
  jacobian_cell<TJ, TP, SURF>(P, i, j, k, c, p, kr, dkr, satv, dsatv, dt, J, M, dl_z, dl_y,
                              dl_x, de, dn, du);
}

// Face-once form (as k_residual_zm): each cell evaluates the derivative
// parts of its right, front and upper faces; the (lo, hi) parts the
// neighbour needs go through shared memory (x, y) or a register (z).
// Shared memory: blockDim.y x (blockDim.x + 1) and (blockDim.y + 1) x
// blockDim.x pairs of TJ.
template <typename TJ, typename TP, bool SURF>
__global__ void __launch_bounds__(256, 3) k_jacobian_zm(DevProblem P, const double *__restrict__ p,
                           const double *__restrict__ kr, const double *__restrict__ dkr,
                           const double *__restrict__ satv, const double *__restrict__ dsatv,
                           double dt, JacOut<TJ> J, PCOut<TP> M, int kchunk) {
  using TA = TJ;
  extern __shared__ __align__(16) unsigned char jz_smem[];
  const int bx = blockDim.x, by = blockDim.y, tx = threadIdx.x, ty = threadIdx.y;
  FaceLH<TA> *sE = reinterpret_cast<FaceLH<TA> *>(jz_smem);  // [by][bx + 1]
  FaceLH<TA> *sN = sE + by * (bx + 1);                         // [by + 1][bx]
  pdl_enter();
  if (P.dtp) dt = *P.dtp;
  const int i = blockIdx.x * bx + tx, j = blockIdx.y * by + ty;
  const int k0 = blockIdx.z * kchunk, k1 = min(P.nz, k0 + kchunk);
  const bool in = i < P.nx && j < P.ny;
  const long long sy = P.nx, sz = (long long)P.nx * P.ny;
  const double rho = P.density, g = P.gravity, drho = 0.0;
  const double ffx = P.dy * P.dz, ffy = P.dx * P.dz;
  double gsw = 0.5 * (g * 0.0 + g * 0.0), gcw = 0.5 * (g * 1.0 + g * 1.0);
  double gss = gsw, gcs = gcw, gse = gsw, gce = gcw, gsn = gsw, gcn = gcw;
  if (SURF && in) {
    if (i > 0) tfg_face_x(P, i - 1, j, gsw, gcw);
    if (j > 0) tfg_face_y(P, i, j - 1, gss, gcs);
    if (i + 1 < P.nx) tfg_face_x(P, i, j, gse, gce);
    if (j + 1 < P.ny) tfg_face_y(P, i, j, gsn, gcn);
  }
  long long c = i + (long long)P.nx * (j + (long long)P.ny * k0);
  FaceLH<TA> dl_z{};
  if (in && k0 > 0 && k0 < k1) {
    const long long q = c - sz;
    FaceDer<TA> d = face_der_z<TA>(P, dt, fb_z(P, q), p[q], p[c], __ldg(P.kz + q), __ldg(P.kz + c),
                                   kr[q] * rho, dkr[q] * rho + kr[q] * drho, kr[c] * rho,
                                   dkr[c] * rho + kr[c] * drho, __ldg(P.zmult + k0 - 1),
                                   __ldg(P.zmult + k0), k0 - 1);
    dl_z = {d.lo, d.hi};
  }
  for (int k = k0; k < k1; k++, c += sz) {
    FaceDer<TA> de{}, dn{}, du{};
    if (in) {
      const double zm = __ldg(P.zmult + k);
      const double pc = p[c];
      const double prod = kr[c] * rho, prod_der = dkr[c] * rho + kr[c] * drho;
      const double kxc = __ldg(P.kx + c), kyc = __ldg(P.ky + c), kzc = __ldg(P.kz + c);
      if (i + 1 < P.nx) {
        const long long q = c + 1;
        de = face_der_xy<TA>(P, dt, fb_x(P, c), ffx, P.dx, P.inv_dx, pc, p[q], kxc,
                             __ldg(P.kx + q), prod, prod_der, kr[q] * rho,
                             dkr[q] * rho + kr[q] * drho, zm, gse, gce);
      }
      if (j + 1 < P.ny) {
        const long long q = c + sy;
        dn = face_der_xy<TA>(P, dt, fb_y(P, c), ffy, P.dy, P.inv_dy, pc, p[q], kyc,
                             __ldg(P.ky + q), prod, prod_der, kr[q] * rho,
                             dkr[q] * rho + kr[q] * drho, zm, gsn, gcn);
      }
      if (k + 1 < P.nz) {
        const long long q = c + sz;
        du = face_der_z<TA>(P, dt, fb_z(P, c), pc, p[q], kzc, __ldg(P.kz + q), prod, prod_der,
                            kr[q] * rho, dkr[q] * rho + kr[q] * drho, zm,
                            __ldg(P.zmult + k + 1), k);
      }
      if (tx == 0 && i > 0) {
        const long long q = c - 1;
        FaceDer<TA> d = face_der_xy<TA>(P, dt, fb_x(P, q), ffx, P.dx, P.inv_dx, p[q], pc,
                                        __ldg(P.kx + q), kxc, kr[q] * rho,
                                        dkr[q] * rho + kr[q] * drho, prod,
                                        prod_der, zm, gsw, gcw);
        sE[ty * (bx + 1)] = {d.lo, d.hi};
      }
      if (ty == 0 && j > 0) {
        const long long q = c - sy;
        FaceDer<TA> d = face_der_xy<TA>(P, dt, fb_y(P, q), ffy, P.dy, P.inv_dy, p[q], pc,
                                        __ldg(P.ky + q), kyc, kr[q] * rho,
                                        dkr[q] * rho + kr[q] * drho, prod,
                                        prod_der, zm, gss, gcs);
        sN[tx] = {d.lo, d.hi};
      }
    }
    sE[ty * (bx + 1) + tx + 1] = {de.lo, de.hi};
    sN[(ty + 1) * bx + tx] = {dn.lo, dn.hi};
    __syncthreads();
    if (in)
      jacobian_cell<TJ, TP, SURF>(P, i, j, k, c, p, kr, dkr, satv, dsatv, dt, J, M, dl_z,
                                  sN[ty * bx + tx], sE[ty * (bx + 1) + tx], de, dn, du);
    dl_z = {du.lo, du.hi};
    __syncthreads();
  }
}

// y = J x (matvec.c:35-330 order: y = 0, then C W E S N L U), FP64 accumulate
template <typename TJ>
__global__ void k_matvec7(int nx, int ny, int nz, JacIn<TJ> J, const double *__restrict__ x,
                          double *__restrict__ y) {
  pdl_enter();
  int i, j, k;
  if (!launch_ijk(nx, ny, nz, i, j, k)) return;
  const long long c = i + (long long)nx * (j + (long long)ny * k);
  const long long sy = nx, sz = (long long)nx * ny;
  double acc = 0.0;
  acc += (double)J.c[c] * x[c];
  acc += (double)J.w[c] * (i > 0 ? x[c - 1] : 0.0);
  acc += (double)J.e[c] * (i + 1 < nx ? x[c + 1] : 0.0);
  acc += (double)J.s[c] * (j > 0 ? x[c - sy] : 0.0);
  acc += (double)J.n[c] * (j + 1 < ny ? x[c + sy] : 0.0);
  acc += (double)J.l[c] * (k > 0 ? x[c - sz] : 0.0);
  acc += (double)J.u[c] * (k + 1 < nz ? x[c + sz] : 0.0);
  y[c] = acc;
}

// ---------------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------------
static inline unsigned blocks_for(long long n, int bs) { return (unsigned)((n + bs - 1) / bs); }

// 3-D launch covering (nx, ny, nz) with `threads` threads per block
static inline void shape(int nx, int ny, int nz, int threads, dim3 &grid, dim3 &block) {
  int bx = 32;
  while (bx < nx && bx < 128) bx *= 2;
  if (bx > threads) bx = threads;
  int by = threads / bx;
  if (by > ny) by = ny;
  block = dim3(bx, by, 1);
  grid = dim3((nx + bx - 1) / bx, (ny + by - 1) / by, nz);
}
// the tuned shape (bx, by) when one is set, else the heuristic
static inline void shape_tuned(int nx, int ny, int nz, int threads, const int tile[2],
                               dim3 &grid, dim3 &block) {
  if (!tile || tile[0] <= 0 || tile[1] <= 0) {
    shape(nx, ny, nz, threads, grid, block);
    return;
  }
  block = dim3(tile[0], tile[1], 1);
  grid = dim3((nx + tile[0] - 1) / tile[0], (ny + tile[1] - 1) / tile[1], nz);
}

void launch_vg_all(const DevProblem &P, const double *p, double *kr, double *dkr, double *sat,
                   double *dsat, cudaStream_t st) {
  launch_pdl(k_vg_all, dim3(blocks_for(P.n, 256)), dim3(256), st, P, p, kr, dkr, sat, dsat);
}

void launch_saturation(const DevProblem &P, const double *p, double *s, cudaStream_t st) {
  launch_pdl(k_saturation, dim3(blocks_for(P.n, 256)), dim3(256), st, P, p, s);
}

// The gather form is the default: on B200 the face-once form runs slower at
// 512x512x50 (0.566 against 0.524 ms for the VG pass plus the residual,
// 0.730 against 0.649 ms for the Jacobian with its VG pass): the shared
// fluxes cost registers and a barrier per plane, and the kernels are bound
// by latency at the occupancy they leave.  PFGPU_RESIDUAL_FACE_ONCE=1 selects
// the face-once form (bitwise the same results).
static bool residual_gather() {
  static const bool on = [] {
    const char *v = getenv("PFGPU_RESIDUAL_FACE_ONCE");
    return !(v && *v == '1');
  }();
  return on;
}

// planes per block of the face-once kernels: enough blocks for about eight
// per SM while each block walks as many planes as that allows
static inline int zm_chunk(const dim3 &g2, int nz) {
  const long long tiles = (long long)g2.x * g2.y;
  long long chunks = (8LL * 148 + tiles - 1) / tiles;
  if (chunks < 1) chunks = 1;
  if (chunks > nz) chunks = nz;
  return (int)((nz + chunks - 1) / chunks);
}

// tile of the face-once kernels: a tuned shape when one is set, else 32 x 8
// (one extra x face per 32 cells and one extra y face per 8)
static inline void zm_shape(int nx, int ny, const int tile[2], dim3 &grid, dim3 &block) {
  int bx = 32, by = 8;
  if (tile && tile[0] > 0 && tile[1] > 0 && tile[0] * tile[1] <= 256) {
    bx = tile[0];
    by = tile[1];
  }
  block = dim3(bx, by, 1);
  grid = dim3((nx + bx - 1) / bx, (ny + by - 1) / by, 1);
}

template <bool SURF, bool VEL>
static void launch_residual_t(const DevProblem &P, const double *p, const double *p_old,
                              const double *s_old, const double *kr, const double *sat,
                              double dt, double *f, cudaStream_t st, const VelOut &vel) {
  dim3 g, b;
  if (residual_gather()) {
    shape_tuned(P.nx, P.ny, P.nz, 256, P.tile[0], g, b);
    launch_pdl(k_residual<SURF, VEL>, dim3(g), dim3(b), st, P, p, p_old, s_old, kr, sat, dt, f,
               vel);
    return;
  }
  zm_shape(P.nx, P.ny, P.tile[0], g, b);
  const int kchunk = zm_chunk(g, P.nz);
  const dim3 gz(g.x, g.y, (P.nz + kchunk - 1) / kchunk);
  const size_t smem = sizeof(double) * ((size_t)b.y * (b.x + 1) + (size_t)(b.y + 1) * b.x);
  launch_pdl_smem(k_residual_zm<SURF, VEL>, gz, b, smem, st, P, p, p_old, s_old, kr, sat, dt, f,
                  vel, kchunk);
}

void launch_residual(const DevProblem &P, const double *p, const double *p_old,
                     const double *s_old, const double *kr, const double *sat, double dt,
                     double *f, cudaStream_t st, const VelOut *vel) {
  const bool surf = P.tfg_xs || P.bc_type[5] == 2 || P.bc_type[5] == 3 || P.bc_type[5] == 4;
  if (vel) {
    if (surf)
      launch_residual_t<true, true>(P, p, p_old, s_old, kr, sat, dt, f, st, *vel);
    else
      launch_residual_t<false, true>(P, p, p_old, s_old, kr, sat, dt, f, st, *vel);
    return;
  }
  if (surf)
    launch_residual_t<true, false>(P, p, p_old, s_old, kr, sat, dt, f, st, VelOut{});
  else
    launch_residual_t<false, false>(P, p, p_old, s_old, kr, sat, dt, f, st, VelOut{});
}

template <typename TJ, typename TP>
void launch_jacobian(const DevProblem &P, const double *p, const double *kr,
                     const double *dkr, const double *sat, const double *dsat, double dt,
                     JacOut<TJ> J, PCOut<TP> M, cudaStream_t st) {
  dim3 g, b;
  const bool surf = P.tfg_xs || P.bc_type[5] == 2 || P.bc_type[5] == 3 || P.bc_type[5] == 4;
  if (residual_gather()) {
    shape_tuned(P.nx, P.ny, P.nz, 128, P.tile[1], g, b);
    if (surf)
      launch_pdl(k_jacobian<TJ, TP, true>, dim3(g), dim3(b), st, P, p, kr, dkr, sat, dsat, dt, J,
                 M);
    else
      launch_pdl(k_jacobian<TJ, TP, false>, dim3(g), dim3(b), st, P, p, kr, dkr, sat, dsat, dt,
                 J, M);
    return;
  }
  zm_shape(P.nx, P.ny, P.tile[1], g, b);
  const int kchunk = zm_chunk(g, P.nz);
  const dim3 gz(g.x, g.y, (P.nz + kchunk - 1) / kchunk);
  const size_t smem = sizeof(FaceLH<TJ>) * ((size_t)b.y * (b.x + 1) + (size_t)(b.y + 1) * b.x);
  if (surf)
    launch_pdl_smem(k_jacobian_zm<TJ, TP, true>, gz, b, smem, st, P, p, kr, dkr, sat, dsat, dt,
                    J, M, kchunk);
  else
    launch_pdl_smem(k_jacobian_zm<TJ, TP, false>, gz, b, smem, st, P, p, kr, dkr, sat, dsat, dt,
                    J, M, kchunk);
}

template <typename TJ>
void launch_matvec7(int nx, int ny, int nz, JacIn<TJ> J, const double *x, double *y,
                    cudaStream_t st, const int *tile) {
  dim3 g, b;
  shape_tuned(nx, ny, nz, 256, tile, g, b);
  launch_pdl(k_matvec7<TJ>, dim3(g), dim3(b), st, nx, ny, nz, J, x, y);
}

template void launch_jacobian<double, double>(const DevProblem &, const double *,
                                              const double *, const double *, const double *,
                                              const double *, double, JacOut<double>,
                                              PCOut<double>, cudaStream_t);
template void launch_jacobian<float, float>(const DevProblem &, const double *, const double *,
                                            const double *, const double *, const double *,
                                            double, JacOut<float>, PCOut<float>, cudaStream_t);
template void launch_matvec7<double>(int, int, int, JacIn<double>, const double *, double *,
                                     cudaStream_t, const int *);
template void launch_matvec7<float>(int, int, int, JacIn<float>, const double *, double *,
                                    cudaStream_t, const int *);

}  // namespace pfgpu
