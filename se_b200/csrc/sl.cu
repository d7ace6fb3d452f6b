// Semi-Lagrangian advection on GLL quadrilateral meshes, sm_100a.
//
// One thread per owned vertex (periodic duplicates are written by their
// partner thread, which is what Field::PeriodicUpdate leaves in the
// reference). Each thread integrates the backward trajectory and gathers the
// (N+1)^2 element block of the field at every stage.
//
// Reference: src/base/Advector.cpp:122-148,181-246,339-349 (PeriodicUpdate, IntegrateRK2,
// FirstOrder, SecondOrder, ExtrapolateVelocities), src/base/Mesh.cpp:109-176
// (GetEl, GlobalToLocal), src/base/Legendre.cpp:145-169 and :293-305
// (ShapeFuncsAtCoord, IsRoot), src/base/Field.cpp:57-76 (InterpLocal/Global).
//
// Parity: coordinates (vertex positions, departure points, element search,
// local coordinates, wrap) use the reference's exact IEEE operation order, so
// that for equal velocities the departure element is bit-identical. The
// cardinal functions use the Lagrange product form with prefix/suffix
// products (no divisions) instead of the reference's P_N' formula; both
// evaluate the same polynomial and agree to a few ulps.
#include "common.cuh"

namespace seg {
namespace {

// ------------------------------------------------------- mesh geometry ----
// Mesh::Mesh vertex coordinate along direction d (src/base/Mesh.cpp:66-71).
__device__ __forceinline__ double vertex_coord(const MeshDev& m, int d, int t) {
  int e = t / m.N;
  double l = m.abcissa[t - e * m.N];
  return xadd(xadd(m.min[d], xmul((double)e, m.dx[d])),
              xmul(xdiv(xadd(l, 1.0), 2.0), m.dx[d]));
}

// Mesh::GetEl along one direction (src/base/Mesh.cpp:109-136). Out-of-mesh
// points (possible only when a trajectory crosses more than one period) are
// clamped to the nearest element and flagged.
__device__ __forceinline__ int get_topo(const MeshDev& m, int d, double c, unsigned* err) {
  double t = xsub(c, m.max[d]);
  if (t >= -1.0e-12 && t <= 1.0e-12) return m.nEls[d] - 1;
  double out = xdiv(xsub(c, m.min[d]), m.dx[d]);
  double integer = trunc(out);
  double frac = out - integer;  // exact
  int topo = (int)integer;
  if (topo > 0 && frac >= -1.0e-12 && frac <= 1.0e-12) topo--;
  if (topo < 0 || topo >= m.nEls[d] || !(out == out)) {
    if (err) atomicOr(err, KERR_DOMAIN);
    topo = topo < 0 || !(out == out) ? 0 : m.nEls[d] - 1;
  }
  return topo;
}

// Mesh::GlobalToLocal along one direction (src/base/Mesh.cpp:163-176).
__device__ __forceinline__ double local_coord(const MeshDev& m, int d, double c, int topo) {
  double l = xsub(xmul(xsub(xsub(c, m.min[d]), xmul((double)topo, m.dx[d])), m.two_over_dx[d]),
                  1.0);
  if (l < -1.0) l = -1.0;
  if (l > +1.0) l = +1.0;
  return l;
}

// Legendre::IsRoot (src/base/Legendre.cpp:293-305): index of the first GLL
// node within 1e-8, or -1.
template <int N>
__device__ __forceinline__ int snap_node(const MeshDev& m, double l) {
  int s = -1;
#pragma unroll
  for (int k = N; k >= 0; k--)
    if (fabs(l - m.abcissa[k]) < 1.0e-8) s = k;
  return s;
}

// GLL cardinal functions at a non-node coordinate: N_j(l) = lambda_j *
// prod_{k != j} (l - x_k), from prefix and suffix products.
template <int N>
__device__ __forceinline__ void cardinal(const MeshDev& m, double l, double* c) {
  double d[N + 1];
#pragma unroll
  for (int k = 0; k <= N; k++) d[k] = l - m.abcissa[k];
  double pre = 1.0;
#pragma unroll
  for (int k = 0; k <= N; k++) {
    c[k] = pre;
    pre *= d[k];
  }
  double suf = 1.0;
#pragma unroll
  for (int k = N; k >= 0; k--) {
    c[k] *= suf * m.lambda[k];
    suf *= d[k];
  }
}

// Advector::PeriodicUpdate (src/base/Advector.cpp:122-134).
__device__ __forceinline__ double wrap(const MeshDev& m, int d, double c) {
  if (c < m.min[d]) c = m.periodic[d] ? xadd(m.span[d], c) : m.min[d];
  if (c > m.max[d]) c = m.periodic[d] ? xadd(m.nspan[d], c) : m.max[d];
  return c;
}

// ----------------------------------------------------------- value types ----
struct V1 {
  double a;
};
struct V2 {
  double a, b;
};
__device__ __forceinline__ V1 vzero(V1) { return {0.0}; }
__device__ __forceinline__ V2 vzero(V2) { return {0.0, 0.0}; }
__device__ __forceinline__ V1 vfma(double s, V1 v, V1 acc) { return {fma(s, v.a, acc.a)}; }
__device__ __forceinline__ V2 vfma(double s, V2 v, V2 acc) {
  return {fma(s, v.a, acc.a), fma(s, v.b, acc.b)};
}

// Sources: the nodal value of a field at vertex k (operator()), the N+1
// values of a vertex row from vertex r0 (row), and an L2 prefetch of the
// line holding vertex k.
//
// Scalar rows of even orders are read as 16-byte pairs: an element row
// starts at an even or odd vertex index, the same for every thread of a warp
// when N is even (the row offsets are multiples of N, the row pitch is odd),
// so a row of 9 values at p=8 is 5 loads instead of 9. Odd orders (whose
// rows start at both parities within a warp) read single values.
struct Scalar {
  typedef V1 T;
  const double* __restrict__ p;
  __device__ __forceinline__ T operator()(int k) const { return {__ldg(p + k)}; }
  template <int N>
  __device__ __forceinline__ void row(int r0, T* v) const {
    const double* q = p + r0;
    if constexpr (N % 2 == 0) {
      // 16-byte alignment from the address itself (q is 8-byte aligned)
      if ((reinterpret_cast<uintptr_t>(q) & 8u) == 0) {
#pragma unroll
        for (int k = 0; k < N; k += 2) {
          const double2 d = __ldg(reinterpret_cast<const double2*>(q + k));
          v[k].a = d.x;
          v[k + 1].a = d.y;
        }
        v[N].a = __ldg(q + N);
      } else {
        v[0].a = __ldg(q);
#pragma unroll
        for (int k = 1; k < N; k += 2) {
          const double2 d = __ldg(reinterpret_cast<const double2*>(q + k));
          v[k].a = d.x;
          v[k + 1].a = d.y;
        }
      }
    } else {
#pragma unroll
      for (int k = 0; k <= N; k++) v[k].a = __ldg(q + k);
    }
  }
  __device__ __forceinline__ void prefetch(int k) const {
    asm volatile("prefetch.global.L2 [%0];" ::"l"(p + k));
  }
};
struct Vec2 {
  typedef V2 T;
  const double2* __restrict__ p;
  __device__ __forceinline__ T operator()(int k) const {
    double2 v = __ldg(p + k);
    return {v.x, v.y};
  }
  template <int N>
  __device__ __forceinline__ void row(int r0, T* v) const {
#pragma unroll
    for (int k = 0; k <= N; k++) v[k] = (*this)(r0 + k);
  }
  __device__ __forceinline__ void prefetch(int k) const {
    asm volatile("prefetch.global.L2 [%0];" ::"l"(p + k));
  }
};
// c0*v + c1*vm with the reference's rounding (Advector::ExtrapolateVelocities,
// src/base/Advector.cpp:339-349): each product rounded, then the sum.
struct Vec2Mix {
  typedef V2 T;
  const double2* __restrict__ v;
  const double2* __restrict__ vm;
  double c0, c1;
  __device__ __forceinline__ T operator()(int k) const {
    double2 a = __ldg(v + k), b = __ldg(vm + k);
    return {xadd(xmul(c0, a.x), xmul(c1, b.x)), xadd(xmul(c0, a.y), xmul(c1, b.y))};
  }
  template <int N>
  __device__ __forceinline__ void row(int r0, T* v) const {
#pragma unroll
    for (int k = 0; k <= N; k++) v[k] = (*this)(r0 + k);
  }
};

// Field::InterpGlobal (src/base/Field.cpp:70-76) at global point (gx, gy).
// Snapped directions reduce to a row, a column or a single vertex; the
// reference sums the same products plus exact zeros.
template <int N, class Src>
__device__ __forceinline__ typename Src::T interp(const MeshDev& m, const Src& src, double gx,
                                                  double gy, int* el_out, unsigned* err) {
  typedef typename Src::T T;
  int tx = get_topo(m, 0, gx, err), ty = get_topo(m, 1, gy, err);
  if (el_out) *el_out = ty * m.nEls[0] + tx;
  double lx = local_coord(m, 0, gx, tx), ly = local_coord(m, 1, gy, ty);
  int sx = snap_node<N>(m, lx), sy = snap_node<N>(m, ly);
  const int nvx = m.nVerts[0];
  const int base = ty * N * nvx + tx * N;
  if (sx >= 0 && sy >= 0) return src(base + sy * nvx + sx);
  double cx[N + 1], cy[N + 1];
  T acc = vzero(T());
  if (sy >= 0) {
    cardinal<N>(m, lx, cx);
    T rv[N + 1];
    src.template row<N>(base + sy * nvx, rv);
#pragma unroll
    for (int i = 0; i <= N; i++) acc = vfma(cx[i], rv[i], acc);
    return acc;
  }
  cardinal<N>(m, ly, cy);
  if (sx >= 0) {
#pragma unroll
    for (int j = 0; j <= N; j++) acc = vfma(cy[j], src(base + j * nvx + sx), acc);
    return acc;
  }
  cardinal<N>(m, lx, cx);
#pragma unroll
  for (int j = 0; j <= N; j++) {
    T rv[N + 1];
    src.template row<N>(base + j * nvx, rv);
    T r = vzero(T());
#pragma unroll
    for (int i = 0; i <= N; i++) r = vfma(cx[i], rv[i], r);
    acc = vfma(cy[j], r, acc);
  }
  return acc;
}

template <class T>
__device__ __forceinline__ void store(double* out, int node, T v);
template <>
__device__ __forceinline__ void store<V1>(double* out, int node, V1 v) {
  out[node] = v.a;
}
template <>
__device__ __forceinline__ void store<V2>(double* out, int node, V2 v) {
  reinterpret_cast<double2*>(out)[node] = make_double2(v.a, v.b);
}

// Write the value of owned vertex (i, j) and of its periodic copies.
template <class T>
__device__ __forceinline__ void store_with_copies(const MeshDev& m, double* out, int i, int j,
                                                  T v) {
  const int nvx = m.nVerts[0], nvy = m.nVerts[1];
  store<T>(out, j * nvx + i, v);
  if (m.periodic[0] && i == 0) store<T>(out, j * nvx + nvx - 1, v);
  if (m.periodic[1] && j == 0) store<T>(out, (nvy - 1) * nvx + i, v);
  if (m.periodic[0] && m.periodic[1] && i == 0 && j == 0) store<T>(out, nvy * nvx - 1, v);
}

// Advector::FirstOrder with IntegrateRK2 (src/base/Advector.cpp:136-148,181-201).
template <int N, class FSrc>
__global__ void __launch_bounds__(256, 2) sl_first_kernel(const MeshDev m, FSrc field,
                                                       const double2* __restrict__ vel,
                                                       double dt, double half_dt,
                                                       double* __restrict__ out,
                                                       int* __restrict__ dep_el,
                                                       double2* __restrict__ dep_xy,
                                                       unsigned* err) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int nvx = m.nVerts[0], nvy = m.nVerts[1];
  const bool owner = i < nvx - m.periodic[0] && j < nvy - m.periodic[1];
  if (i >= nvx || j >= nvy || (!owner && !dep_el)) return;
  Vec2 v{vel};
  // the tracer near this vertex, where most departure points land: its
  // lines start their way from HBM while the velocity is interpolated
  field.prefetch(j * nvx + i);
  const double ox = vertex_coord(m, 0, i), oy = vertex_coord(m, 1, j);
  V2 u = interp<N>(m, v, ox, oy, nullptr, err);
  double xh = wrap(m, 0, xsub(ox, xmul(half_dt, u.a)));
  double yh = wrap(m, 1, xsub(oy, xmul(half_dt, u.b)));
  u = interp<N>(m, v, xh, yh, nullptr, err);
  const double xd = wrap(m, 0, xsub(ox, xmul(dt, u.a)));
  const double yd = wrap(m, 1, xsub(oy, xmul(dt, u.b)));
  int el;
  typename FSrc::T val = interp<N>(m, field, xd, yd, &el, err);
  if (dep_el) {
    dep_el[j * nvx + i] = el;
    if (dep_xy) dep_xy[j * nvx + i] = make_double2(xd, yd);
  }
  if (owner) store_with_copies(m, out, i, j, val);
}

// Advector::SecondOrder (src/base/Advector.cpp:203-246) with the
// extrapolated velocities formed on the fly at each gathered vertex.
template <int N, class FSrc>
__global__ void __launch_bounds__(256, 2) sl_second_kernel(const MeshDev m, FSrc field,
                                                        FSrc field_prev,
                                                        const double2* __restrict__ vel,
                                                        const double2* __restrict__ vel_prev,
                                                        double dt, double half_dt,
                                                        double* __restrict__ out,
                                                        int* __restrict__ dep_el,
                                                        double2* __restrict__ dep_xy,
                                                        unsigned* err) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int nvx = m.nVerts[0], nvy = m.nVerts[1];
  const bool owner = i < nvx - m.periodic[0] && j < nvy - m.periodic[1];
  if (i >= nvx || j >= nvy || (!owner && !dep_el)) return;
  const Vec2Mix plus_one{vel, vel_prev, 2.0, -1.0};
  const Vec2Mix plus_half{vel, vel_prev, 1.5, -0.5};
  const Vec2Mix minus_half{vel, vel_prev, 0.5, 0.5};
  const Vec2 v{vel};
  const double ox = vertex_coord(m, 0, i), oy = vertex_coord(m, 1, j);
  V2 u = interp<N>(m, plus_one, ox, oy, nullptr, err);
  double xh = wrap(m, 0, xsub(ox, xmul(half_dt, u.a)));
  double yh = wrap(m, 1, xsub(oy, xmul(half_dt, u.b)));
  u = interp<N>(m, plus_half, xh, yh, nullptr, err);
  const double x1 = wrap(m, 0, xsub(ox, xmul(dt, u.a)));
  const double y1 = wrap(m, 1, xsub(oy, xmul(dt, u.b)));
  u = interp<N>(m, v, x1, y1, nullptr, err);
  xh = wrap(m, 0, xsub(x1, xmul(half_dt, u.a)));
  yh = wrap(m, 1, xsub(y1, xmul(half_dt, u.b)));
  u = interp<N>(m, minus_half, xh, yh, nullptr, err);
  const double x2 = wrap(m, 0, xsub(x1, xmul(dt, u.a)));
  const double y2 = wrap(m, 1, xsub(y1, xmul(dt, u.b)));
  int el1, el2;
  typename FSrc::T p1 = interp<N>(m, field, x1, y1, &el1, err);
  typename FSrc::T p2 = interp<N>(m, field_prev, x2, y2, &el2, err);
  if (dep_el) {
    const int nv = nvx * nvy;
    dep_el[j * nvx + i] = el1;
    dep_el[nv + j * nvx + i] = el2;
    if (dep_xy) {
      dep_xy[j * nvx + i] = make_double2(x1, y1);
      dep_xy[nv + j * nvx + i] = make_double2(x2, y2);
    }
  }
  if (owner) {
    // fieldSL = 2 psi(x1) - 0.5 psiPrev(x2) (src/base/Advector.cpp:236-240)
    typename FSrc::T r;
    double* rp = reinterpret_cast<double*>(&r);
    const double* a = reinterpret_cast<const double*>(&p1);
    const double* b = reinterpret_cast<const double*>(&p2);
#pragma unroll
    for (int d = 0; d < (int)(sizeof(r) / sizeof(double)); d++)
      rp[d] = xsub(xmul(2.0, a[d]), xmul(0.5, b[d]));
    store_with_copies(m, out, i, j, r);
  }
}

template <int N>
cudaError_t launch_sl_n(const MeshDev& m, int ndofs, const double* field, const double* vel,
                        const double* field_prev, const double* vel_prev, double dt, double* out,
                        int* dep_el, double* dep_xy, unsigned* err, cudaStream_t s) {
  // a warp covers 8 x 4 vertices, about one element: its departure points
  // fall in fewer element blocks than a row of 32 vertices' do
  dim3 block(8, 32);
  dim3 grid((m.nVerts[0] + 7) / 8, (m.nVerts[1] + 31) / 32);
  const double half_dt = 0.5 * dt;
  const double2* v = reinterpret_cast<const double2*>(vel);
  const double2* vm = reinterpret_cast<const double2*>(vel_prev);
  double2* dxy = reinterpret_cast<double2*>(dep_xy);
  if (!field_prev) {
    if (ndofs == 1)
      sl_first_kernel<N, Scalar><<<grid, block, 0, s>>>(m, Scalar{field}, v, dt, half_dt, out,
                                                         dep_el, dxy, err);
    else
      sl_first_kernel<N, Vec2><<<grid, block, 0, s>>>(
          m, Vec2{reinterpret_cast<const double2*>(field)}, v, dt, half_dt, out, dep_el, dxy,
          err);
  } else {
    if (ndofs == 1)
      sl_second_kernel<N, Scalar><<<grid, block, 0, s>>>(m, Scalar{field}, Scalar{field_prev},
                                                          v, vm, dt, half_dt, out, dep_el, dxy,
                                                          err);
    else
      sl_second_kernel<N, Vec2><<<grid, block, 0, s>>>(
          m, Vec2{reinterpret_cast<const double2*>(field)},
          Vec2{reinterpret_cast<const double2*>(field_prev)}, v, vm, dt, half_dt, out, dep_el,
          dxy, err);
  }
  return cudaGetLastError();
}

// ------------------------------------------------ point queries (tests) ----
__global__ void global_to_local_kernel(const MeshDev m, const double2* __restrict__ pts,
                                       int npts, int* el, double2* lc) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= npts) return;
  double2 p = pts[k];
  int tx = get_topo(m, 0, p.x, nullptr), ty = get_topo(m, 1, p.y, nullptr);
  el[k] = ty * m.nEls[0] + tx;
  lc[k] = make_double2(local_coord(m, 0, p.x, tx), local_coord(m, 1, p.y, ty));
}

template <int N>
__global__ void interp_points_kernel(const MeshDev m, int ndofs, const double* __restrict__ vals,
                                     const double2* __restrict__ pts, int npts, double* out) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= npts) return;
  double2 p = pts[k];
  if (ndofs == 1) {
    V1 r = interp<N>(m, Scalar{vals}, p.x, p.y, nullptr, nullptr);
    out[k] = r.a;
  } else {
    V2 r = interp<N>(m, Vec2{reinterpret_cast<const double2*>(vals)}, p.x, p.y, nullptr, nullptr);
    out[2 * k] = r.a;
    out[2 * k + 1] = r.b;
  }
}

__global__ void periodic_update_kernel(const MeshDev m, int ndofs, double* vals) {
  const int nvx = m.nVerts[0], nvy = m.nVerts[1];
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  // rows: copy column 0 -> nvx-1; then columns: row 0 -> nvy-1 (incl. corner)
  if (m.periodic[0] && k < nvy)
    for (int d = 0; d < ndofs; d++)
      vals[(size_t)(k * nvx + nvx - 1) * ndofs + d] = vals[(size_t)(k * nvx) * ndofs + d];
}
__global__ void periodic_update_rows_kernel(const MeshDev m, int ndofs, double* vals) {
  const int nvx = m.nVerts[0], nvy = m.nVerts[1];
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (m.periodic[1] && k < nvx)
    for (int d = 0; d < ndofs; d++)
      vals[(size_t)((nvy - 1) * nvx + k) * ndofs + d] = vals[(size_t)k * ndofs + d];
}

// Fixed-order block reduction of two sums; deterministic.
template <int B>
__device__ __forceinline__ void block_sum2(double& a, double& b) {
  __shared__ double sa[B / 32], sb[B / 32];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    a += __shfl_down_sync(0xffffffffu, a, o);
    b += __shfl_down_sync(0xffffffffu, b, o);
  }
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0) {
    sa[w] = a;
    sb[w] = b;
  }
  __syncthreads();
  if (w == 0) {
    a = l < B / 32 ? sa[l] : 0.0;
    b = l < B / 32 ? sb[l] : 0.0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      a += __shfl_down_sync(0xffffffffu, a, o);
      b += __shfl_down_sync(0xffffffffu, b, o);
    }
  }
}

// Element quadrature sums with the affine Jacobian (hx/2)(hy/2): one block
// per group of elements, partials summed in a second pass in fixed order.
__global__ void __launch_bounds__(256) quadrature_kernel(const MeshDev m, int ndofs, int dof,
                                                         const double* __restrict__ a,
                                                         const double* __restrict__ b,
                                                         double* partial) {
  const int n = m.N + 1, nn = n * n;
  const int nel = m.nEls[0] * m.nEls[1];
  const double detj = (0.5 * m.dx[0]) * (0.5 * m.dx[1]);
  double s0 = 0.0, s1 = 0.0;
  for (long q = (long)blockIdx.x * blockDim.x + threadIdx.x; q < (long)nel * nn;
       q += (long)gridDim.x * blockDim.x) {
    int el = (int)(q / nn), pt = (int)(q - (long)el * nn);
    int px = pt % n, py = pt / n;
    int ex = el % m.nEls[0], ey = el / m.nEls[0];
    int node = (ey * m.N + py) * m.nVerts[0] + ex * m.N + px;
    double wq = detj * (m.w[px] * m.w[py]);
    double va = a[(size_t)node * ndofs + dof];
    if (b) {
      double vb = b[(size_t)node * ndofs + dof];
      s0 += wq * (va - vb) * (va - vb);
      s1 += wq * vb * vb;
    } else {
      s0 += wq * va;
    }
  }
  block_sum2<256>(s0, s1);
  if (threadIdx.x == 0) {
    partial[2 * blockIdx.x] = s0;
    partial[2 * blockIdx.x + 1] = s1;
  }
}
__global__ void __launch_bounds__(256) sum_partials_kernel(const double* partial, int np,
                                                           double* out2) {
  double s0 = 0.0, s1 = 0.0;
  for (int k = threadIdx.x; k < np; k += blockDim.x) {
    s0 += partial[2 * k];
    s1 += partial[2 * k + 1];
  }
  block_sum2<256>(s0, s1);
  if (threadIdx.x == 0) {
    out2[0] = s0;
    out2[1] = s1;
  }
}
__global__ void __launch_bounds__(256) max_speed_kernel(int nv, const double2* __restrict__ vel,
                                                        double* partial) {
  double mx = 0.0;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nv; k += gridDim.x * blockDim.x) {
    double2 v = vel[k];
    double s = v.x * v.x + v.y * v.y;
    mx = fmax(mx, s);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_down_sync(0xffffffffu, mx, o));
  __shared__ double sm[8];
  if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = mx;
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < 8; w++) mx = fmax(mx, sm[w]);
    partial[blockIdx.x] = mx;
  }
}
__global__ void max_partials_kernel(const double* partial, int np, double* out) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    double mx = 0.0;
    for (int k = 0; k < np; k++) mx = fmax(mx, partial[k]);
    *out = mx;
  }
}

// TwoLayerQGEqn::GenVel / QuasiGeostrophicEqn::GenVel
// (src/qg/TwoLayerQGEqn.cpp:335-352, src/qg/QuasiGeostrophicEqn.cpp:207-223):
// vel = (-d psi/dy, d psi/dx) at every vertex, each derivative from
// Field::InterpDerivsGlobal (src/base/Field.cpp:96-118) in the element that
// GetEl picks for the vertex. A vertex's local coordinates are GLL nodes in
// both directions, so Mesh::ShapeFuncDerivsAtCoord gives d/dxi = dC[xi][j] on
// the node's row and d/deta = dC[yi][j] on its column, exact zeros elsewhere;
// the Jacobian, its inverse and the sums are formed in the reference's order
// over the row and column entries (the zero products leave the sums as they
// are), with exactly rounded operations.
// d/dx, d/dy of component `dof` of an ndofs-component field at vertex (i, j)
// (returns false if the vertex's local coordinates did not snap to nodes).
template <int N>
__device__ __forceinline__ bool vertex_derivs(const MeshDev& m, const double* __restrict__ vals,
                                              int ndofs, int dof, int i, int j, double& dx,
                                              double& dy, unsigned* err) {
  constexpr int n = N + 1;
  const int nvx = m.nVerts[0];
  const double gx = vertex_coord(m, 0, i), gy = vertex_coord(m, 1, j);
  const int tx = get_topo(m, 0, gx, err), ty = get_topo(m, 1, gy, err);
  const int xi = snap_node<N>(m, local_coord(m, 0, gx, tx));
  const int yi = snap_node<N>(m, local_coord(m, 1, gy, ty));
  if (xi < 0 || yi < 0) return false;
  const int base = ty * N * nvx + tx * N;
  const double* rowd = m.dC + xi * n;  // d/dxi of the cardinals along the row
  const double* cold = m.dC + yi * n;  // d/deta along the column
  // Jacobian: J00 = sum g0 x, J01 = sum g0 y, J10 = sum g1 x, J11 = sum g1 y
  double J00 = 0.0, J01 = 0.0, J10 = 0.0, J11 = 0.0;
  const double yrow = vertex_coord(m, 1, ty * N + yi), xcol = vertex_coord(m, 0, tx * N + xi);
#pragma unroll
  for (int b = 0; b < n; b++) {
    const double xb = vertex_coord(m, 0, tx * N + b);
    J00 = xadd(J00, xmul(rowd[b], xb));
    J01 = xadd(J01, xmul(rowd[b], yrow));
  }
#pragma unroll
  for (int b = 0; b < n; b++) {
    const double yb = vertex_coord(m, 1, ty * N + b);
    J10 = xadd(J10, xmul(cold[b], xcol));
    J11 = xadd(J11, xmul(cold[b], yb));
  }
  const double det = xsub(xmul(J00, J11), xmul(J01, J10));
  const double I00 = xdiv(J11, det), I11 = xdiv(J00, det);
  const double I01 = xdiv(-J01, det), I10 = xdiv(-J10, det);
  // sums over the element's nodes in node order (row yj, column xj); only
  // the node's row and column contribute
  double sx = 0.0, sy = 0.0;
#pragma unroll
  for (int yj = 0; yj < n; yj++) {
    if (yj == yi) {
#pragma unroll
      for (int xj = 0; xj < n; xj++) {
        const double g0 = rowd[xj], g1 = xj == xi ? cold[yj] : 0.0;
        const double p = __ldg(vals + (size_t)(base + yj * nvx + xj) * ndofs + dof);
        const double tx_ = xadd(xmul(g0, I00), xmul(g1, I01));
        const double ty_ = xadd(xmul(g0, I10), xmul(g1, I11));
        sx = xadd(sx, xmul(tx_, p));
        sy = xadd(sy, xmul(ty_, p));
      }
    } else {
      const double g1 = cold[yj];
      const double p = __ldg(vals + (size_t)(base + yj * nvx + xi) * ndofs + dof);
      sx = xadd(sx, xmul(xmul(g1, I01), p));
      sy = xadd(sy, xmul(xmul(g1, I11), p));
    }
  }
  dx = sx;
  dy = sy;
  return true;
}

// TwoLayerQGEqn::GenVel / QuasiGeostrophicEqn::GenVel
// (src/qg/TwoLayerQGEqn.cpp:335-352, src/qg/QuasiGeostrophicEqn.cpp:207-223):
// vel = (-d psi/dy, d psi/dx) at every vertex, each derivative from
// Field::InterpDerivsGlobal (src/base/Field.cpp:96-118) in the element that
// GetEl picks for the vertex. A vertex's local coordinates are GLL nodes in
// both directions, so Mesh::ShapeFuncDerivsAtCoord gives d/dxi = dC[xi][j] on
// the node's row and d/deta = dC[yi][j] on its column, exact zeros elsewhere;
// the Jacobian, its inverse and the sums are formed in the reference's order
// over the row and column entries (the zero products leave the sums as they
// are), with exactly rounded operations.
template <int N>
__global__ void gen_vel_kernel(const MeshDev m, const double* __restrict__ psi,
                               double2* __restrict__ vel, unsigned* err) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  if (i >= m.nVerts[0] || j >= m.nVerts[1]) return;
  double dx, dy;
  if (!vertex_derivs<N>(m, psi, 1, 0, i, j, dx, dy, err)) {  // a vertex always lies on a node
    if (err) atomicOr(err, (unsigned)KERR_BAD_CONFIG);
    return;
  }
  vel[j * m.nVerts[0] + i] = make_double2(-dy, dx);
}

// NavierStokesEqn's pressure step (src/ns/NavierStokesEqn.cpp:63-85 and
// :109-131): kind 0: out[v] = du/dx + dv/dy of the 2-component field a;
// kind 2: the same times 1.5 times 10.0 (the second-order step's factor, as
// the reference writes it); kind 1: out[v] = a[v] - dt grad p (a 2
// components, p scalar).
template <int N>
__global__ void ns_pressure_kernel(const MeshDev m, int kind, const double* __restrict__ a,
                                   const double* __restrict__ p, double dt,
                                   double* __restrict__ out, unsigned* err) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  if (i >= m.nVerts[0] || j >= m.nVerts[1]) return;
  const int v = j * m.nVerts[0] + i;
  if (kind != 1) {
    double ux, uy, vx, vy;
    if (!vertex_derivs<N>(m, a, 2, 0, i, j, ux, uy, err) ||
        !vertex_derivs<N>(m, a, 2, 1, i, j, vx, vy, err)) {
      if (err) atomicOr(err, (unsigned)KERR_BAD_CONFIG);
      return;
    }
    out[v] = kind == 2 ? (ux + vy) * 1.5 * 10.0 : ux + vy;
  } else {
    double px, py;
    if (!vertex_derivs<N>(m, p, 1, 0, i, j, px, py, err)) {
      if (err) atomicOr(err, (unsigned)KERR_BAD_CONFIG);
      return;
    }
    out[2 * v] = a[2 * v] - dt * px;
    out[2 * v + 1] = a[2 * v + 1] - dt * py;
  }
}

// Component `dof` of a 2-component field to / from a scalar field.
__global__ void component_kernel(int nv, int to_scalar, int dof, double* __restrict__ two,
                                 double* __restrict__ one) {
  const int v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= nv) return;
  if (to_scalar)
    one[v] = two[2 * v + dof];
  else
    two[2 * v + dof] = one[v];
}

// ------------------------------------------------- two-layer QG pieces ----
// TwoLayerQGEqn::GenPV (src/qg/TwoLayerQGEqn.cpp:326-333):
// alpha = omega + F (psi_j - psi_i) + beta y at every vertex.
__global__ void gen_pv_kernel(const MeshDev m, const double* __restrict__ omega,
                              const double* __restrict__ psi_i, const double* __restrict__ psi_j,
                              double F, double beta, double* __restrict__ alpha) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y;
  if (i >= m.nVerts[0]) return;
  const int v = j * m.nVerts[0] + i;
  const double y = vertex_coord(m, 1, j);
  alpha[v] = omega[v] + F * (psi_j[v] - psi_i[v]) + beta * y;
}

// The step's pointwise combinations (src/qg/TwoLayerQGEqn.cpp:186-232,
// 264-323): kind 0: out0 = a - b (Helmholtz right-hand side); kind 1:
// out0 = a + b + dF t - cb y (Poisson right-hand side); kind 2: the stream
// functions and vorticities from t (baroclinic) and c (barotropic):
// out0 = psi1, out1 = psi2, out2 = omega1, out3 = omega2.
__global__ void qg_combine_kernel(const MeshDev m, int kind, const double* __restrict__ a,
                                  const double* __restrict__ b, const double* __restrict__ t,
                                  const double* __restrict__ c, double F1, double F2, double cb,
                                  double* out0, double* out1, double* out2, double* out3) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y;
  if (i >= m.nVerts[0]) return;
  const int v = j * m.nVerts[0] + i;
  const double y = vertex_coord(m, 1, j);
  if (kind == 0) {
    out0[v] = a[v] - b[v];
  } else if (kind == 1) {
    out0[v] = a[v] + b[v] + (F1 - F2) * t[v] - cb * y;
  } else {
    const double p1 = 0.5 * (t[v] + c[v]), p2 = 0.5 * (c[v] - t[v]);
    out0[v] = p1;
    out1[v] = p2;
    out2[v] = a[v] - F1 * (p2 - p1) - cb * y;
    out3[v] = b[v] - F2 * (p1 - p2) - cb * y;
  }
}

// Element options of a vertex along one direction: (element, node) pairs in
// ascending element order (a shared vertex belongs to two elements; the
// periodic seam joins the last element's node N to vertex 0).
__device__ __forceinline__ int vertex_elements(const MeshDev& m, int d, int g, int* e, int* a) {
  const int N = m.N, nE = m.nEls[d];
  int k = 0;
  const int eo = g / N, ao = g - eo * N;
  if (ao == 0) {
    if (eo > 0) {
      e[k] = eo - 1;
      a[k++] = N;
    } else if (m.periodic[d]) {
      e[k] = nE - 1;  // sorted below
      a[k++] = N;
    }
  }
  if (eo < nE) {
    e[k] = eo;
    a[k++] = ao;
  }
  if (k == 2 && e[0] > e[1]) {  // periodic seam: keep ascending element order
    int te = e[0], ta = a[0];
    e[0] = e[1];
    a[0] = a[1];
    e[1] = te;
    a[1] = ta;
  }
  return k;
}

// TwoLayerQGEqn::SolveQ (src/qg/TwoLayerQGEqn.cpp:396-418) with the
// DissipationRHS vector (:435-463) of one layer, per unknown: gathers the
// element contributions at the unknown's vertex in element order,
//   detJ w (q + dt rF t - dt Ei omegaHat - dt rF tau_e)
//   - dt nu detJ sum_pt w_pt grad N_k(pt) . grad omegaHat(pt),
// with grad omegaHat at a point taken as at its vertex in the element GetEl
// picks (grad: omegaHat's GenVel field, (-d/dy, d/dx) at every vertex);
// divides by the assembled PV mass a detJ w (the GLL mass matrix is
// diagonal) and writes the unknown's vertex and its periodic copies
// (Vector::UpdateField).
__global__ void qg_solve_q_kernel(const MeshDev m, Dir dxd, Dir dyd, int G0, double dt,
                                  const double* __restrict__ q, const double* __restrict__ tau,
                                  const double* __restrict__ omh, const double2* __restrict__ grad,
                                  const double* __restrict__ tau_e, double rF, double Ei, double nu,
                                  double a, double* __restrict__ alpha) {
  const int ux = blockIdx.x * blockDim.x + threadIdx.x, uy = blockIdx.y;
  if (ux >= G0) return;
  const int N = m.N, n = N + 1, nvx = m.nVerts[0], nvy = m.nVerts[1];
  const int gx = ux + dxd.lo, gy = uy + dyd.lo;
  const int v = gy * nvx + gx;
  const double det = (0.5 * m.dx[0]) * (0.5 * m.dx[1]);
  const double sx = 2.0 / m.dx[0], sy = 2.0 / m.dx[1];
  int ex[2], ax[2], ey[2], ay[2];
  const int kx = vertex_elements(m, 0, gx, ex, ax), ky = vertex_elements(m, 1, gy, ey, ay);
  const double own = q[v] + dt * rF * tau[v] - dt * Ei * omh[v] - dt * rF * tau_e[v];
  double f = 0.0, dsum = 0.0;
  for (int jy = 0; jy < ky; jy++)      // element rows ascending ...
    for (int jx = 0; jx < kx; jx++) {  // ... then columns: ascending element index
      const int ex_ = ex[jx], ax_ = ax[jx], ey_ = ey[jy], ay_ = ay[jy];
      const double wk = m.w[ax_] * m.w[ay_];
      double gsum = 0.0;
      // d/dx of cardinal ax_ along the node's row, d/dy along its column
      for (int p = 0; p < n; p++) {
        const int vx = (ey_ * N + ay_) * nvx + ex_ * N + p;
        gsum += sx * m.w[ay_] * m.w[p] * m.dC[p * n + ax_] * grad[vx].y;   // d/dx
        const int vy = (ey_ * N + p) * nvx + ex_ * N + ax_;
        gsum -= sy * m.w[ax_] * m.w[p] * m.dC[p * n + ay_] * grad[vy].x;   // d/dy = -(.x)
      }
      f += det * wk * own - dt * nu * det * gsum;
      dsum += a * det * wk;
    }
  const double x = f / dsum;
  alpha[v] = x;
  const bool cx = m.periodic[0] && gx == 0, cy = m.periodic[1] && gy == 0;
  if (cx) alpha[gy * nvx + nvx - 1] = x;
  if (cy) alpha[(nvy - 1) * nvx + gx] = x;
  if (cx && cy) alpha[nvy * nvx - 1] = x;
}

}  // namespace

// Dispatch a runtime polynomial order onto the compile-time one (NN).
#define SE_DISPATCH_N(N, ...)                     \
  switch (N) {                                    \
    case 2: { constexpr int NN = 2; __VA_ARGS__; }   \
    case 3: { constexpr int NN = 3; __VA_ARGS__; }   \
    case 4: { constexpr int NN = 4; __VA_ARGS__; }   \
    case 5: { constexpr int NN = 5; __VA_ARGS__; }   \
    case 6: { constexpr int NN = 6; __VA_ARGS__; }   \
    case 7: { constexpr int NN = 7; __VA_ARGS__; }   \
    case 8: { constexpr int NN = 8; __VA_ARGS__; }   \
    case 9: { constexpr int NN = 9; __VA_ARGS__; }   \
    case 10: { constexpr int NN = 10; __VA_ARGS__; } \
    case 11: { constexpr int NN = 11; __VA_ARGS__; } \
    case 12: { constexpr int NN = 12; __VA_ARGS__; } \
    default: return cudaErrorInvalidValue;        \
  }

cudaError_t launch_sl(const MeshDev& m, int ndofs, const double* field, const double* vel,
                      const double* field_prev, const double* vel_prev, double dt, double* out,
                      int* dep_el, double* dep_xy, unsigned* err, cudaStream_t s) {
  if (m.N < 3) return cudaErrorInvalidValue;
  SE_DISPATCH_N(m.N, return launch_sl_n<NN>(m, ndofs, field, vel, field_prev, vel_prev, dt, out,
                                            dep_el, dep_xy, err, s));
}

cudaError_t launch_ns_pressure(const MeshDev& m, int kind, const double* a, const double* p,
                               double dt, double* out, unsigned* err, cudaStream_t s) {
  const dim3 block(32, 8);
  const dim3 grid((m.nVerts[0] + 31) / 32, (m.nVerts[1] + 7) / 8);
  SE_DISPATCH_N(m.N, {
    ns_pressure_kernel<NN><<<grid, block, 0, s>>>(m, kind, a, p, dt, out, err);
    return cudaGetLastError();
  });
}

cudaError_t launch_component(int nv, int to_scalar, int dof, double* two, double* one,
                             cudaStream_t s) {
  component_kernel<<<(nv + 255) / 256, 256, 0, s>>>(nv, to_scalar, dof, two, one);
  return cudaGetLastError();
}

cudaError_t launch_gen_pv(const MeshDev& m, const double* omega, const double* psi_i,
                          const double* psi_j, double F, double beta, double* alpha, cudaStream_t s) {
  const dim3 grid((m.nVerts[0] + 255) / 256, m.nVerts[1]);
  gen_pv_kernel<<<grid, 256, 0, s>>>(m, omega, psi_i, psi_j, F, beta, alpha);
  return cudaGetLastError();
}

cudaError_t launch_qg_combine(const MeshDev& m, int kind, const double* a, const double* b,
                              const double* t, const double* c, double F1, double F2, double cb,
                              double* out0, double* out1, double* out2, double* out3,
                              cudaStream_t s) {
  const dim3 grid((m.nVerts[0] + 255) / 256, m.nVerts[1]);
  qg_combine_kernel<<<grid, 256, 0, s>>>(m, kind, a, b, t, c, F1, F2, cb, out0, out1, out2, out3);
  return cudaGetLastError();
}

cudaError_t launch_qg_solve_q(const MeshDev& m, const Dir& dx, const Dir& dy, double dt,
                              const double* q, const double* tau, const double* omh,
                              const double* grad, const double* tau_e, double rF, double Ei,
                              double nu, double a, double* alpha, cudaStream_t s) {
  const int G0 = dx.hi - dx.lo, G1 = dy.hi - dy.lo;
  if (G0 <= 0 || G1 <= 0) return cudaSuccess;
  const dim3 grid((G0 + 127) / 128, G1);
  qg_solve_q_kernel<<<grid, 128, 0, s>>>(m, dx, dy, G0, dt, q, tau, omh,
                                         reinterpret_cast<const double2*>(grad), tau_e, rF, Ei, nu,
                                         a, alpha);
  return cudaGetLastError();
}

cudaError_t launch_gen_vel(const MeshDev& m, const double* psi, double* vel, unsigned* err,
                           cudaStream_t s) {
  const dim3 block(32, 8);
  const dim3 grid((m.nVerts[0] + 31) / 32, (m.nVerts[1] + 7) / 8);
  SE_DISPATCH_N(m.N, {
    gen_vel_kernel<NN><<<grid, block, 0, s>>>(m, psi, reinterpret_cast<double2*>(vel), err);
    return cudaGetLastError();
  });
}

cudaError_t launch_global_to_local(const MeshDev& m, const double* pts, int npts, int* el,
                                   double* lc, cudaStream_t s) {
  if (npts <= 0) return cudaSuccess;
  global_to_local_kernel<<<(npts + 255) / 256, 256, 0, s>>>(
      m, reinterpret_cast<const double2*>(pts), npts, el, reinterpret_cast<double2*>(lc));
  return cudaGetLastError();
}

cudaError_t launch_interp_global(const MeshDev& m, int ndofs, const double* vals,
                                 const double* pts, int npts, double* out, cudaStream_t s) {
  if (npts <= 0) return cudaSuccess;
  SE_DISPATCH_N(m.N, {
    interp_points_kernel<NN><<<(npts + 127) / 128, 128, 0, s>>>(
        m, ndofs, vals, reinterpret_cast<const double2*>(pts), npts, out);
    return cudaGetLastError();
  });
}

cudaError_t launch_periodic_update(const MeshDev& m, int ndofs, double* vals, cudaStream_t s) {
  if (m.periodic[0])
    periodic_update_kernel<<<(m.nVerts[1] + 255) / 256, 256, 0, s>>>(m, ndofs, vals);
  if (m.periodic[1])
    periodic_update_rows_kernel<<<(m.nVerts[0] + 255) / 256, 256, 0, s>>>(m, ndofs, vals);
  return cudaGetLastError();
}

cudaError_t launch_quadrature(const MeshDev& m, int ndofs, int dof, const double* a,
                              const double* b, double* scratch, int nscratch, double* out2,
                              cudaStream_t s) {
  long work = (long)m.nEls[0] * m.nEls[1] * (m.N + 1) * (m.N + 1);
  int blocks = (int)((work + 255) / 256);
  if (blocks > nscratch / 2) blocks = nscratch / 2;
  if (blocks < 1) return cudaErrorInvalidValue;
  quadrature_kernel<<<blocks, 256, 0, s>>>(m, ndofs, dof, a, b, scratch);
  sum_partials_kernel<<<1, 256, 0, s>>>(scratch, blocks, out2);
  return cudaGetLastError();
}

cudaError_t launch_max_speed_sq(int nv, const double* vel, double* scratch, int nscratch,
                                double* out, cudaStream_t s) {
  int blocks = (nv + 255) / 256;
  if (blocks > nscratch) blocks = nscratch;
  if (blocks < 1) return cudaErrorInvalidValue;
  max_speed_kernel<<<blocks, 256, 0, s>>>(nv, reinterpret_cast<const double2*>(vel), scratch);
  max_partials_kernel<<<1, 32, 0, s>>>(scratch, blocks, out);
  return cudaGetLastError();
}

}  // namespace seg
