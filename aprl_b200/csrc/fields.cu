// fields.cu -- grid kernels of the step: Cowan-z Faraday with the CPML
// magnetic correction, the zero-current Ampere preview with the CPML
// electric correction, PEC termination and inlet overwrite, the commit
// E^{n+1} = E* - dt/eps0 J, and the moving-window plane insertion.
//
// E, B and the CPML histories are binary64 in every mode, and every
// expression keeps the reference's operation order; the library is compiled
// without FMA contraction, so these kernels reproduce the reference's
// translation units bit for bit.  The kernels are templated on the type F of
// the current J (double, or float in the FP32-mixed mode), which only the
// commit reads.
#include "common.cuh"
#include "dd.cuh"
#include "fields.cuh"

namespace aprl_gpu {

// electricValue (src/eb_field.cpp:350-417) under the moving window: x/y
// PEC parity extension, z halo planes (lower = inlet reference plane,
// upper = the last rank's zero plane).
template <class F>
__device__ __forceinline__ double electric_value(const CowanArgs<F>& a, int c, int i, int j,
                                                 int k) {
  const int nxc = a.g.nx + (c != 0), nyc = a.g.ny + (c != 1), nzc = a.g.nz + (c != 2);
  double sign = 1.0;
  if (i < 0) {
    if (c == 0) i = 0; else { i = -i; sign = -sign; }
  } else if (i >= nxc) {
    if (c == 0) i = nxc - 1; else { i = 2 * (nxc - 1) - i; sign = -sign; }
  }
  if (j < 0) {
    if (c == 1) j = 0; else { j = -j; sign = -sign; }
  } else if (j >= nyc) {
    if (c == 1) j = nyc - 1; else { j = 2 * (nyc - 1) - j; sign = -sign; }
  }
  if (k < 0)
    return sign * a.lower[c][APRL_BOUNDED(a.g.status, (size_t)j * nxc + i, (size_t)nxc * nyc, 10 + c)];
  if (k >= nzc) return sign * 0.0;
  return sign * a.e[c][APRL_BOUNDED(a.g.status,
                                    ((size_t)ring(k, a.g.zb_e[c], nzc) * nyc + j) * nxc + i,
                                    (size_t)nxc * nyc * nzc, 13 + c)];
}

// transformedCorrection (src/eb_cpml.cpp:131-138).
__device__ __forceinline__ double cpml_correction(const CpmlAxis& ax, int index,
                                                  double difference, double* history) {
  const double psi = ax.decay[index] * *history + ax.drive[index] * difference;
  *history = psi;
  return ax.inverse_kappa_minus_one[index] * difference + psi;
}

__device__ __forceinline__ double* history_at(const CpmlHistory& h, int slot, int k, int zbase,
                                              int row_index, DeviceStatus* status) {
  (void)status;
  return h.data + APRL_BOUNDED(status,
                               ((size_t)slot * h.layers + ring(k, zbase, h.layers)) * h.row +
                                   row_index,
                               (size_t)h.slots * h.layers * h.row, 16);
}

// advanceMagneticCowan (src/eb_field.cpp:488-558) fused with
// EBConvolutionalPML::afterMagneticUpdate (src/eb_cpml.cpp:406-468).
//
// A block owns a TX x TY tile of (i, j) columns and marches a chunk of z
// planes.  The three E components of planes k-1, k, k+1 live in a shared
// memory ring, one (TX+2) x (TY+2) tile each, loaded once per plane through
// electricValue's parity/halo rules.  Every smoothed difference (the
// 9-point smoothedElectric of src/eb_field.cpp:419-486: alpha*centre, the
// four beta edge samples, the four delta corners) is then evaluated from
// shared memory in the reference's order, so the FP64 update is
// bit-identical to the reference.  Each B node is updated by the
// curl, then by its CPML terms in the reference's term order (0,2,1),
// (1,2,0), (2,1,0), (2,0,1), reusing the curl's smoothed difference.
constexpr int kTX = kCowanTileX, kTY = kCowanTileY;

struct ETile {
  double v[3][3][kTY + 2][kTX + 2];  // [component][plane slot][y][x]
};

// Ring slots of the tile planes k-1, k, k+1 of the current z-march step,
// rotated by one per step (no modular arithmetic in the stencil).
struct PlaneSlots {
  int s[3];
};

__device__ __forceinline__ double tile_at(const ETile& t, int c, int li, int lj, int dk,
                                          const PlaneSlots& ps) {
  return t.v[c][ps.s[dk + 1]][lj][li];
}

// smoothedElectric from the tile: centre (li, lj) in tile coordinates, dk
// the plane offset (-1..1) from the marching plane; every offset is a
// compile-time constant after inlining, so the plane choice is a register.
template <class F>
__device__ __forceinline__ double tile_smoothed(const ETile& t, const CowanArgs<F>& a, int c,
                                                int d, int li, int lj, int dk,
                                                const PlaneSlots& ps) {
  const int ta = (d + 1) % 3, tb = (d + 2) % 3;
  const double delta = d == 0 ? a.delta_yz : (d == 1 ? a.delta_zx : a.delta_xy);
  const int p[3] = {li, lj, dk};
  double result = a.alpha[d] * tile_at(t, c, li, lj, dk, ps);
#pragma unroll
  for (int dir = -1; dir <= 1; dir += 2) {
    int qa[3] = {p[0], p[1], p[2]}, qb[3] = {p[0], p[1], p[2]};
    qa[ta] += dir;
    qb[tb] += dir;
    result += a.beta[ta] * tile_at(t, c, qa[0], qa[1], qa[2], ps);
    result += a.beta[tb] * tile_at(t, c, qb[0], qb[1], qb[2], ps);
  }
#pragma unroll
  for (int da = -1; da <= 1; da += 2)
#pragma unroll
    for (int db = -1; db <= 1; db += 2) {
      int q[3] = {p[0], p[1], p[2]};
      q[ta] += da;
      q[tb] += db;
      result += delta * tile_at(t, c, q[0], q[1], q[2], ps);
    }
  return result;
}

// Fills one plane of the tile.  Only coordinates within one cell of a
// component's index range are ever read by the smoothing (the reference's
// own reach); tile points farther out, which exist only where a small grid
// ends inside a tile, are stored as zero and never used.
template <class F>
__device__ __forceinline__ void load_plane(ETile& t, const CowanArgs<F>& a, int k, int slot,
                                           int i0, int j0) {
  constexpr int W = kTX + 2, H = kTY + 2, N = W * H, T = kTX * kTY, R = (N + T - 1) / T;
  const int tid = threadIdx.y * kTX + threadIdx.x;
  // A tile whose rim lies inside every component's index range, on a plane
  // inside every component's z range, needs none of electricValue's parity
  // and halo rules: its values are read straight from E.
  const bool interior = i0 >= 1 && i0 + kTX <= a.g.nx - 1 && j0 >= 1 &&
                        j0 + kTY <= a.g.ny - 1 && k >= 0 && k < a.g.nz;
  // All of a thread's loads are issued before any shared-memory store, so
  // their latencies overlap instead of adding up.
  double v[3][R];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    const int nxc = a.g.nx + (c != 0), nyc = a.g.ny + (c != 1), nzc = a.g.nz + (c != 2);
    const double* plane =
        interior ? a.e[c] + (size_t)ring(k, a.g.zb_e[c], nzc) * nyc * nxc : nullptr;
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const int n = tid + r * T;
      double x = 0.0;
      if (n < N) {
        const int ii = n % W, jj = n / W;
        const int i = i0 - 1 + ii, j = j0 - 1 + jj;
        if (interior)
          x = plane[APRL_BOUNDED(a.g.status, (size_t)j * nxc + i, (size_t)nxc * nyc, 19 + c)];
        else if (!(i < -1 || i > nxc || j < -1 || j > nyc))
          x = electric_value(a, c, i, j, k);
      }
      v[c][r] = x;
    }
  }
#pragma unroll
  for (int c = 0; c < 3; ++c)
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const int n = tid + r * T;
      if (n < N) t.v[c][slot][n / W][n % W] = v[c][r];
    }
}

template <class F>
__global__ void __launch_bounds__(kTX * kTY, APRL_COWAN_MIN_BLOCKS)
    cowan_magnetic_kernel(CowanArgs<F> a) {
  __shared__ ETile t;
  const GridT<F>& g = a.g;
  const int i0 = blockIdx.x * kTX, j0 = blockIdx.y * kTY;
  const int i = i0 + threadIdx.x, j = j0 + threadIdx.y;
  const int k0 = blockIdx.z * a.chunk;
  const int k1 = min(k0 + a.chunk, g.nz + 1);
  const double dtdx = g.dt / g.dx, dtdy = g.dt / g.dy, dtdz = g.dt / g.dz;
  const int li = threadIdx.x + 1, lj = threadIdx.y + 1;
  PlaneSlots ps = {{0, 1, 2}};
  load_plane(t, a, k0 - 1, ps.s[0], i0, j0);
  load_plane(t, a, k0, ps.s[1], i0, j0);
  // The column's CPML slots are the same on every plane of the march.
  const bool column = i <= g.nx && j <= g.ny;
  const int slot_x = column && i < g.nx ? a.mx.ordinal[i] : -1;
  const int slot_y = column && j < g.ny ? a.my.ordinal[j] : -1;
  // The z differences smooth within one plane (x and y neighbours), so the
  // smoothed Ey and Ex of plane k+1 are, bit for bit, the plane-k operands
  // of the next step: carried in registers instead of evaluated again.
  double ey_above = 0.0, ex_above = 0.0;
  for (int k = k0; k < k1; ++k) {
    load_plane(t, a, k + 1, ps.s[2], i0, j0);
    // The node's three B values are read before the first B store (which
    // may alias them as far as the compiler knows).
    const bool has_bx = column && j < g.ny && k < g.nz;
    const bool has_by = column && i < g.nx && k < g.nz;
    const bool has_bz = column && i < g.nx && j < g.ny;
    double* const bx = has_bx ? &g.b[0][b_index(g, 0, i, j, k)] : nullptr;
    double* const by = has_by ? &g.b[1][b_index(g, 1, i, j, k)] : nullptr;
    double* const bz = has_bz ? &g.b[2][b_index(g, 2, i, j, k)] : nullptr;
    const double bx_old = has_bx ? *bx : 0.0;
    const double by_old = has_by ? *by : 0.0;
    const double bz_old = has_bz ? *bz : 0.0;
    __syncthreads();
    if (i <= g.nx && j <= g.ny) {
      if (j < g.ny && k < g.nz) {  // Bx (nx+1, ny, nz)
        const double dEzDy = tile_smoothed(t, a, 2, 1, li, lj + 1, 0, ps) -
                             tile_smoothed(t, a, 2, 1, li, lj, 0, ps);
        const double ey_here = k > k0 ? ey_above : tile_smoothed(t, a, 1, 2, li, lj, 0, ps);
        ey_above = tile_smoothed(t, a, 1, 2, li, lj, 1, ps);
        const double dEyDz = ey_above - ey_here;
        double v = bx_old - (dtdy * dEzDy - dtdz * dEyDz);
        const int s = slot_y;
        if (s >= 0)
          v += -1.0 * dtdy * cpml_correction(a.my, j, dEzDy,
                                             history_at(a.h[0], s, k, g.zb_b[0], i, g.status));
        *bx = v;
      }
      if (i < g.nx && k < g.nz) {  // By (nx, ny+1, nz)
        const double ex_here = k > k0 ? ex_above : tile_smoothed(t, a, 0, 2, li, lj, 0, ps);
        ex_above = tile_smoothed(t, a, 0, 2, li, lj, 1, ps);
        const double dExDz = ex_above - ex_here;
        const double dEzDx = tile_smoothed(t, a, 2, 0, li + 1, lj, 0, ps) -
                             tile_smoothed(t, a, 2, 0, li, lj, 0, ps);
        double v = by_old - (dtdz * dExDz - dtdx * dEzDx);
        const int s = slot_x;
        if (s >= 0)
          v += 1.0 * dtdx * cpml_correction(a.mx, i, dEzDx,
                                            history_at(a.h[1], s, k, g.zb_b[1], j, g.status));
        *by = v;
      }
      if (i < g.nx && j < g.ny) {  // Bz (nx, ny, nz+1)
        const double dEyDx = tile_smoothed(t, a, 1, 0, li + 1, lj, 0, ps) -
                             tile_smoothed(t, a, 1, 0, li, lj, 0, ps);
        const double dExDy = tile_smoothed(t, a, 0, 1, li, lj + 1, 0, ps) -
                             tile_smoothed(t, a, 0, 1, li, lj, 0, ps);
        double v = bz_old - (dtdx * dEyDx - dtdy * dExDy);
        const int sx = slot_x;
        if (sx >= 0)
          v += -1.0 * dtdx * cpml_correction(a.mx, i, dEyDx,
                                             history_at(a.h[2], sx, k, g.zb_b[2], j, g.status));
        const int sy = slot_y;
        if (sy >= 0)
          v += 1.0 * dtdy * cpml_correction(a.my, j, dExDy,
                                            history_at(a.h[3], sy, k, g.zb_b[2], i, g.status));
        *bz = v;
      }
    }
    __syncthreads();
    ps = PlaneSlots{{ps.s[1], ps.s[2], ps.s[0]}};
  }
}

template <class F>
__device__ __forceinline__ double bval(const GridT<F>& g, int c, int i, int j, int k) {
  return g.b[c][b_index(g, c, i, j, k)];
}

// advanceElectric with J = 0 (src/eb_field.cpp:582-627) followed by the
// moving-window boundary (src/moving_window_fields.cpp:254-293): the CPML
// electric terms (src/eb_cpml.cpp:470-539; the convolution histories are
// advanced here once, exactly as the later commit would advance them from
// the same B), PEC on the x/y faces, and the inlet Ex/Ey overwrite at k=0.
// Reads E^n from e_old, writes E* to e_star.
template <class F>
__device__ __forceinline__ void preview_orbit(const PreviewArgs<F>& a, int c, size_t n,
                                              double e_star, double e_old) {
  // orbit_sum_kernel without current: S = W(E* + E^n), the same expression.
  if (a.orbit_float)
    static_cast<float*>(a.orbit[c])[n] = float(e_star + e_old);
  else
    static_cast<double*>(a.orbit[c])[n] = e_star + e_old;
}

template <class F>
__global__ void electric_preview_kernel(PreviewArgs<F> a) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = blockIdx.z;
  const GridT<F>& g = a.g;
  if (i > g.nx || j > g.ny || k > g.nz) return;
  const double curl = g.dt / (kMu0 * kEpsilon0);
  const double cx = curl / g.dx, cy = curl / g.dy, cz = curl / g.dz;
  // Every E and B read of the node is issued before its first store (the
  // stores may alias them as far as the compiler knows), so their latencies
  // overlap; each difference below is formed from the same two values as
  // before, in the same order.
  const bool has_x = i < g.nx, has_y = j < g.ny, has_z = k < g.nz;
  const bool x_row = has_x && j >= 1 && j < g.ny;     // Ex: y difference of Bz
  const bool x_curl = x_row && k >= 1 && k < g.nz;    // Ex: the whole curl
  const bool y_row = has_y && i >= 1 && i < g.nx;     // Ey: x difference of Bz
  const bool y_curl = y_row && k >= 1 && k < g.nz;    // Ey: the whole curl
  const bool z_inner = has_z && i >= 1 && i < g.nx && j >= 1 && j < g.ny;
  const size_t n0 = has_x ? e_index(g, 0, i, j, k) : 0;
  const size_t n1 = has_y ? e_index(g, 1, i, j, k) : 0;
  const size_t n2 = has_z ? e_index(g, 2, i, j, k) : 0;
  const double old0 = has_x ? g.e_old[0][n0] : 0.0;
  const double old1 = has_y ? g.e_old[1][n1] : 0.0;
  const double old2 = has_z ? g.e_old[2][n2] : 0.0;
  const double bz = x_row || y_row ? bval(g, 2, i, j, k) : 0.0;
  const double bz_j = x_row ? bval(g, 2, i, j - 1, k) : 0.0;
  const double bz_i = y_row ? bval(g, 2, i - 1, j, k) : 0.0;
  const double by = x_curl || z_inner ? bval(g, 1, i, j, k) : 0.0;
  const double by_k = x_curl ? bval(g, 1, i, j, k - 1) : 0.0;
  const double by_i = z_inner ? bval(g, 1, i - 1, j, k) : 0.0;
  const double bx = y_curl || z_inner ? bval(g, 0, i, j, k) : 0.0;
  const double bx_k = y_curl ? bval(g, 0, i, j, k - 1) : 0.0;
  const double bx_j = z_inner ? bval(g, 0, i, j - 1, k) : 0.0;
  if (has_x) {  // Ex (nx, ny+1, nz+1)
    double v = old0;
    if (x_curl) v += cy * (bz - bz_j) - cz * (by - by_k);
    if (x_row) {
      const int s = a.ey_prof.ordinal[j];
      if (s >= 0) {
        const double diff = bz - bz_j;
        v += 1.0 * cy * cpml_correction(a.ey_prof, j, diff,
                                        history_at(a.h[0], s, k, g.zb_e[0], i, g.status));
      }
    }
    if (j == 0 || j == g.ny) v = 0.0;
    if (k == 0) {
      if (a.pre_inlet[0])
        a.pre_inlet[0][APRL_BOUNDED(g.status, (size_t)j * g.nx + i, (size_t)g.nx * (g.ny + 1), 22)] = v;
      v = inlet_value(a.inlet, 0, i, j);
    }
    g.e_star[0][n0] = v;
    if (a.orbit[0]) preview_orbit(a, 0, n0, v, old0);
  }
  if (has_y) {  // Ey (nx+1, ny, nz+1)
    double v = old1;
    if (y_curl) v += cz * (bx - bx_k) - cx * (bz - bz_i);
    if (y_row) {
      const int s = a.ex_prof.ordinal[i];
      if (s >= 0) {
        const double diff = bz - bz_i;
        v += -1.0 * cx * cpml_correction(a.ex_prof, i, diff,
                                         history_at(a.h[1], s, k, g.zb_e[1], j, g.status));
      }
    }
    if (i == 0 || i == g.nx) v = 0.0;
    if (k == 0) {
      if (a.pre_inlet[1])
        a.pre_inlet[1][APRL_BOUNDED(g.status, (size_t)j * (g.nx + 1) + i,
                                    (size_t)(g.nx + 1) * g.ny, 23)] = v;
      v = inlet_value(a.inlet, 1, i, j);
    }
    g.e_star[1][n1] = v;
    if (a.orbit[0]) preview_orbit(a, 1, n1, v, old1);
  }
  if (has_z) {  // Ez (nx+1, ny+1, nz)
    double v = old2;
    if (z_inner) v += cx * (by - by_i) - cy * (bx - bx_j);
    if (z_inner) {
      const int sx = a.ex_prof.ordinal[i];
      if (sx >= 0) {
        const double diff = by - by_i;
        v += 1.0 * cx * cpml_correction(a.ex_prof, i, diff,
                                        history_at(a.h[2], sx, k, g.zb_e[2], j, g.status));
      }
      const int sy = a.ey_prof.ordinal[j];
      if (sy >= 0) {
        const double diff = bx - bx_j;
        v += -1.0 * cy * cpml_correction(a.ey_prof, j, diff,
                                         history_at(a.h[3], sy, k, g.zb_e[2], i, g.status));
      }
    }
    if (i == 0 || i == g.nx || j == 0 || j == g.ny) v = 0.0;
    g.e_star[2][n2] = v;
    if (a.orbit[0]) preview_orbit(a, 2, n2, v, old2);
  }
}

// commitConservativeElectric (src/simulation_source_coupling.cpp:61-65): the
// previewed boundary already holds the committed CPML/PEC/inlet values, so
// E^{n+1} = E* - dt/eps0 J on the applyCurrentSource mask, in place.
template <class F>
__global__ void electric_commit_kernel(GridT<F> g) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = blockIdx.z;
  if (i > g.nx || j > g.ny || k > g.nz) return;
  // The three J reads are issued before the first update of E* (which may
  // alias them as far as the compiler knows), so their latencies overlap.
  F jc[3];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    jc[c] = F(0.);
    if (i < e_nx(g, c) && j < e_ny(g, c) && k < e_nz(g, c) && current_mask(g, c, i, j, k))
      jc[c] = g.j[c][j_index(g, c, i, j, k)];
  }
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    if (jc[c] != F(0.)) {
      // binary64 J: g.jcoef is -dt/eps0 itself.  A binary32 J is widened and
      // scaled by the binary64 coefficient.
      const double jcoef =
          sizeof(F) == sizeof(double) ? (double)g.jcoef : -1. * g.dt / kEpsilon0;
      g.e_star[c][e_index(g, c, i, j, k)] += jcoef * (double)jc[c];
    }
  }
}

// Boundary::begin lower halo planes (src/moving_window_fields.cpp:206-210):
// reference(a, i, j, offset-1, step) for Ex, Ey, Ez.
__global__ void inlet_lower_kernel(InletPlaneArgs a) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int c = blockIdx.z;
  const int nxc = a.nx + (c != 0), nyc = a.ny + (c != 1);
  if (i >= nxc || j >= nyc) return;
  a.out[c][(size_t)j * nxc + i] = inlet_value(a.inlet, c, i, j);
}

__global__ void inlet_complete_kernel(InletCompleteArgs a) {
  const DGrid& g = a.g;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  if (i <= a.cx || i >= g.nx - a.cx || j <= a.cy || j >= g.ny - a.cy) return;
  // The reference evaluates this in long double; double-double here.
  const DD dex = two_sum(g.e_old[0][e_index(g, 0, i, j, 1)], -g.e_old[0][e_index(g, 0, i - 1, j, 1)]);
  const DD dey = two_sum(g.e_old[1][e_index(g, 1, i, j, 1)], -g.e_old[1][e_index(g, 1, i, j - 1, 1)]);
  const DD divxy = dd_add(dd_div(dex, g.dx), dd_div(dey, g.dy));
  const DD source = dd_div(DD{a.rho[(size_t)j * (g.nx + 1) + i], 0.}, kEpsilon0);
  const DD change = dd_mul(dd_add(divxy, dd_neg(source)), g.dz);
  const double value = dd_value(dd_add(DD{g.e_old[2][e_index(g, 2, i, j, 1)], 0.}, change));
  if (!isfinite(value)) {
    raise_error(a.status, kErrInletField, (unsigned long long)((size_t)j * (g.nx + 1) + i));
    return;
  }
  g.e_old[2][e_index(g, 2, i, j, 0)] = value;
}

__global__ void inlet_halo_kernel(InletHaloArgs a) {
  const DGrid& g = a.g;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  if (i <= a.cx || i >= g.nx - a.cx || j <= a.cy || j >= g.ny - a.cy) return;
  a.lower_ez[(size_t)j * (g.nx + 1) + i] -=
      g.e_old[2][e_index(g, 2, i, j, 0)] - inlet_value(a.inlet, 2, i, j);
}

// MovingWindowFields::shift plane insertion (src/moving_window_fields.cpp:
// 470-517) on the ring: after the bases moved down by one, logical plane 0
// (the dropped upper plane's storage) receives reference(a, i, j, offset,
// step) for E and B, and every CPML history gets a zero layer at k = 0.
template <class F>
__global__ void shift_insert_kernel(ShiftArgs<F> a) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int c = blockIdx.z;  // 0..5 fields, 6..13 histories
  const GridT<F>& g = a.g;
  if (c < 3) {
    const int nxc = e_nx(g, c), nyc = e_ny(g, c);
    if (i >= nxc || j >= nyc) return;
    g.e_old[c][e_index(g, c, i, j, 0)] = inlet_value(a.inlet, c, i, j);
  } else if (c < 6) {
    const int b = c - 3;
    const int nxc = b_nx(g, b), nyc = b_ny(g, b);
    if (i >= nxc || j >= nyc) return;
    g.b[b][b_index(g, b, i, j, 0)] = inlet_value(a.inlet, c, i, j);
  } else {
    const CpmlHistory& h = a.h[c - 6];
    // i runs over the row, j over the slots.
    if (i >= h.row || j >= h.slots) return;
    *history_at(h, j, 0, a.history_base[c - 6], i, g.status) = 0.0;
  }
}

// The orbit sum the electric gathers read, one pass per trial:
// S = E_new + E^n at every E node, with E_new = E* - dt/eps0 J on the
// applyCurrentSource mask (with_current) or E* (the first-trial guess, before
// any current).  In binary64 this is exactly the sum the orbit-averaged
// gather forms node by node (Impl::electric, src/source_coupling.cpp:31-39),
// so the gather is unchanged bit for bit; W = float rounds it once.
template <class W>
__global__ void orbit_sum_kernel(GridT<double> g, W* s0, W* s1, W* s2, int with_current) {
  if (trial_skipped(g)) return;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = blockIdx.z;
  W* s[3] = {s0, s1, s2};
  // Every read of the node is issued before its first store (which may
  // alias them as far as the compiler knows), so their latencies overlap.
  bool in[3];
  size_t n[3];
  double star[3], old[3], jc[3];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    in[c] = i < e_nx(g, c) && j < e_ny(g, c) && k < e_nz(g, c);
    n[c] = in[c] ? e_index(g, c, i, j, k) : 0;
    star[c] = in[c] ? g.e_star[c][n[c]] : 0.;
    old[c] = in[c] ? g.e_old[c][n[c]] : 0.;
    jc[c] = in[c] && with_current && current_mask(g, c, i, j, k)
                ? g.j[c][j_index(g, c, i, j, k)]
                : 0.;
  }
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    if (!in[c]) continue;
    double v = star[c];
    if (jc[c] != 0.) v += g.jcoef * jc[c];
    s[c][n[c]] = W(v + old[c]);
  }
}

// Binary32 copy of B (same ring layout) for the FP32-mixed gathers; one
// launch for the three components (blockIdx.y).
__global__ void b_shadow_kernel(BShadowArgs a) {
  const int c = blockIdx.y;
  // Select by branch: a run-time index into the parameter arrays would copy
  // them to local memory in every thread.
  const double* b = c == 0 ? a.b[0] : (c == 1 ? a.b[1] : a.b[2]);
  float* out = c == 0 ? a.out[0] : (c == 1 ? a.out[1] : a.out[2]);
  const long long n = c == 0 ? a.n[0] : (c == 1 ? a.n[1] : a.n[2]);
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = (float)b[i];
}

// Lab detector field plane (src/lab_detectors.cpp:39-99, 2836-2905).
__device__ __forceinline__ void interp_axis(double lattice, int size, int* lower,
                                            double* fraction) {
  if (lattice <= 0.0) {
    *lower = 0;
    *fraction = 0.0;
  } else if (lattice >= (double)(size - 1)) {
    *lower = size - 2;
    *fraction = 1.0;
  } else {
    *lower = (int)floor(lattice);
    *fraction = lattice - (double)*lower;
  }
}

template <class F>
__device__ double detector_component(const GridT<F>& g, int comp, double lx, double ly, int zl,
                                     double zf) {
  const bool electric = comp < 3;
  const int c = comp % 3;
  const int nxc = electric ? e_nx(g, c) : b_nx(g, c);
  const int nyc = electric ? e_ny(g, c) : b_ny(g, c);
  int xl, yl;
  double xf, yf;
  interp_axis(lx, nxc, &xl, &xf);
  interp_axis(ly, nyc, &yl, &yf);
  double value = 0.0;
  for (int cz = 0; cz < 2; ++cz) {
    const double wz = cz ? zf : 1.0 - zf;
    if (wz == 0.0) continue;
    for (int b = 0; b < 2; ++b)
      for (int a = 0; a < 2; ++a) {
        const double wx = a ? xf : 1.0 - xf;
        const double wy = b ? yf : 1.0 - yf;
        const double v = electric ? g.e_old[c][e_index(g, c, xl + a, yl + b, zl + cz)]
                                  : g.b[c][b_index(g, c, xl + a, yl + b, zl + cz)];
        value += wx * wy * wz * v;
      }
  }
  return value;
}

template <class F>
__global__ void detector_plane_kernel(DetectorArgs<F> a) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const GridT<F>& g = a.g;
  if (i >= g.nx || j >= g.ny) return;
  const double py = a.origin_xy[1] + ((double)j + 0.5) * g.dy;
  const double y = (py - a.origin_xy[1]) / g.dy;
  const double px = a.origin_xy[0] + ((double)i + 0.5) * g.dx;
  const double x = (px - a.origin_xy[0]) / g.dx;
  double eb[3], bb[3];
  eb[0] = detector_component(g, 0, x - 0.5, y, a.vertex_lower, a.vertex_fraction);
  eb[1] = detector_component(g, 1, x, y - 0.5, a.vertex_lower, a.vertex_fraction);
  eb[2] = detector_component(g, 2, x, y, a.half_lower, a.half_fraction);
  bb[0] = detector_component(g, 3, x, y - 0.5, a.half_lower, a.half_fraction);
  bb[1] = detector_component(g, 4, x - 0.5, y, a.half_lower, a.half_fraction);
  bb[2] = detector_component(g, 5, x - 0.5, y - 0.5, a.vertex_lower, a.vertex_fraction);
  // fieldsBoxToLab (src/boostframe.cpp:275-285)
  const DFrame& f = a.frame;
  double* o = a.out + 6 * ((size_t)j * g.nx + i);
  o[0] = fma(f.gamma_beta * kC, bb[1], f.gamma * eb[0]);
  o[1] = fma(-f.gamma_beta * kC, bb[0], f.gamma * eb[1]);
  o[2] = eb[2];
  o[3] = fma(-f.gamma_beta / kC, eb[1], f.gamma * bb[0]);
  o[4] = fma(f.gamma_beta / kC, eb[0], f.gamma * bb[1]);
  o[5] = bb[2];
}

// Built for binary64 J (both modes of this library).
#define APRL_FIELD_KERNELS(F)                                                  \
  template __global__ void cowan_magnetic_kernel<F>(CowanArgs<F>);            \
  template __global__ void electric_preview_kernel<F>(PreviewArgs<F>);        \
  template __global__ void electric_commit_kernel<F>(GridT<F>);               \
  template __global__ void shift_insert_kernel<F>(ShiftArgs<F>);              \
  template __global__ void detector_plane_kernel<F>(DetectorArgs<F>);
APRL_FIELD_KERNELS(double)
template __global__ void orbit_sum_kernel<double>(GridT<double>, double*, double*, double*, int);
template __global__ void orbit_sum_kernel<float>(GridT<double>, float*, float*, float*, int);
#undef APRL_FIELD_KERNELS

// TransverseReferenceCurrent::prepare's values (src/transverse_reference_current.cpp:
// 52-58): curl_z of the reference B at every target point and reference plane,
// ((By(i,j,k) - By(i-1,j,k))/dx - (Bx(i,j,k) - Bx(i,j-1,k))/dy)/mu0.
__global__ void surface_prepare_kernel(SurfaceArgs a) {
  const long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= a.count * a.planes) return;
  const long long k = n / a.count, p = n % a.count;
  const size_t i = a.points[2 * p], j = a.points[2 * p + 1];
  // native reference layouts: Bx (nx+1, ny, planes), By (nx, ny+1, planes)
  const size_t bx0 = ((size_t)k * a.ny + j) * (a.nx + 1) + i;
  const size_t bx1 = ((size_t)k * a.ny + j - 1) * (a.nx + 1) + i;
  const size_t by0 = ((size_t)k * (a.ny + 1) + j) * a.nx + i;
  const double v = ((a.by[by0] - a.by[by0 - 1]) / a.dx - (a.bx[bx0] - a.bx[bx1]) / a.dy) / kMu0;
  if (!isfinite(v)) raise_error(a.status, kErrSurfaceCurrent, (unsigned long long)n);
  a.table[n] = v;
}

// TransverseReferenceCurrent::apply (src/transverse_reference_current.cpp:104-118):
// Jz(i, j, k) += the lerp of the prepared planes at offset + k - beta*step.
__global__ void surface_add_kernel(SurfaceArgs a) {
  const long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const DGrid& g = a.g;
  if (trial_skipped(g) || n >= a.count * g.nz) return;
  const int k = (int)(n / a.count);
  const long long p = n % a.count;
  const double z = static_cast<double>(a.offset + k) - a.beta * static_cast<double>(a.step);
  const long long lo = (long long)floor(z);
  const long long hi = lo + 1 < a.planes ? lo + 1 : a.planes - 1;
  const double fraction = z - (double)lo;
  const double low = a.table[lo * a.count + p], high = a.table[hi * a.count + p];
  const double value = fraction == 0. ? low : (1. - fraction) * low + fraction * high;
  const int i = (int)a.points[2 * p], j = (int)a.points[2 * p + 1];
  g.j[2][j_index(g, 2, i, j, k)] += value;
}

}  // namespace aprl_gpu
