// The reference's frictional boundary inside the persistent forward step
// (contact.py:77-1015): per local/global iteration one semismooth Newton step
// on the Fischer-Burmeister function of every registered vertex against a
// planar, spherical or mesh boundary, an isotropic Coulomb stick/slip
// update, and the position correction x = A^{-1} b + sum_j A^{-1} e_j f_j
// over the candidates that carry force.
//
// Layout: the panel P = A^{-1}[:, nodes] is [n][K] row-major, so the
// correction of particle i reads one contiguous row; B = P[nodes] is [K][K].
// Frames, Delassus matrix W_ij = (n_i . n_j) B_ij and the regularisation are
// frozen at the step start. The Newton section (compaction, response, right
// hand side, coupled block and its factorisation, multiplier and friction
// updates) runs in one block between two team barriers for up to
// kTeamContacts registered vertices, and spread over the team with a blocked
// Cholesky for more (the floor face of a block: hundreds).
#pragma once

#include <cfloat>

#include "pd_device.cuh"
#include "pd_geometry.cuh"

namespace pdb200 {

constexpr int kBoundaryPlanar = 0;
constexpr int kBoundarySpherical = 1;
constexpr int kBoundaryMesh = 2;

__device__ __forceinline__ double fb_solved(const StepArgs& a, int i, int c) {
  // A^{-1} b of this iteration: the product itself, or the refined delta plus x_prev.
  return a.refine ? a.x[3 * i + c] + a.prev[3 * i + c] : a.x[3 * i + c];
}

// boundary_gap / boundary_normal (contact.py:77-98), in the reference's operation order.
__device__ __forceinline__ double fb_gap(const FrictionArgs& f, V3<double> p) {
  const double* q = f.params;
  if (f.kind == kBoundaryPlanar) {
    const double norm = sqrt(q[0] * q[0] + q[1] * q[1] + q[2] * q[2]);
    return (p.x * (q[0] / norm) + p.y * (q[1] / norm) + p.z * (q[2] / norm)) + q[3] / norm;
  }
  const V3<double> d = p - v3<double>(q[0], q[1], q[2]);
  return sqrt(dot(d, d)) - q[3];
}

__device__ __forceinline__ V3<double> fb_normal(const FrictionArgs& f, V3<double> p) {
  const double* q = f.params;
  if (f.kind == kBoundaryPlanar) {
    const double norm = sqrt(q[0] * q[0] + q[1] * q[1] + q[2] * q[2]);
    return v3<double>(q[0] / norm, q[1] / norm, q[2] / norm);
  }
  const V3<double> d = p - v3<double>(q[0], q[1], q[2]);
  const double norm = sqrt(dot(d, d));
  return v3<double>(d.x / norm, d.y / norm, d.z / norm);
}

// Closest point on the surface opposite `node` (faces_right below the split
// index, faces_left otherwise) by one warp: lanes take every 32nd face, the
// smallest distance wins and, among equal distances, the first face, as in
// the reference's sequential loop (contact.py:101-138). Results in every lane.
__device__ inline void fb_mesh_closest(const FrictionArgs& f, V3<double> p, int node, const double* x,
                                       V3<double>& closest, V3<double>& face_normal, double& dist2) {
  const int lane = threadIdx.x & 31;
  int first = f.left_count, last = f.face_count;
  if (node >= f.split) {
    first = 0;
    last = f.left_count;
  }
  double best = INFINITY;
  int best_face = last;
  V3<double> point = v3<double>(0.0, 0.0, 0.0);
  for (int k = first + lane; k < last; k += 32) {
    const int* face = f.faces + 3 * k;
    const TrianglePoint hit = closest_point(p, load3d(x, face[0]), load3d(x, face[1]), load3d(x, face[2]));
    const V3<double> d = p - hit.point;
    const double d2 = dot3(d, d);
    if (d2 < best) {
      best = d2;
      best_face = k;
      point = hit.point;
    }
  }
  double smallest = best;
#pragma unroll
  for (int offset = 16; offset > 0; offset >>= 1) smallest = fmin(smallest, __shfl_xor_sync(0xffffffffu, smallest, offset));
  int owner = best == smallest ? best_face : last;
#pragma unroll
  for (int offset = 16; offset > 0; offset >>= 1) owner = min(owner, __shfl_xor_sync(0xffffffffu, owner, offset));
  const unsigned holders = __ballot_sync(0xffffffffu, best_face == owner && best == smallest);
  const int source = holders != 0u ? __ffs(holders) - 1 : 0;
  closest = v3<double>(__shfl_sync(0xffffffffu, point.x, source), __shfl_sync(0xffffffffu, point.y, source),
                       __shfl_sync(0xffffffffu, point.z, source));
  dist2 = smallest;
  face_normal = v3<double>(0.0, 0.0, 1.0);
  if (owner < last) {
    const int* face = f.faces + 3 * owner;
    const V3<double> a = load3d(x, face[0]);
    const V3<double> n = cross(load3d(x, face[1]) - a, load3d(x, face[2]) - a);
    const double norm = sqrt(dot(n, n));
    if (norm > DBL_EPSILON) face_normal = v3<double>(n.x / norm, n.y / norm, n.z / norm);
  }
}

// mesh_direction (contact.py:141-147): from the closest point toward p, or the face normal on it.
__device__ __forceinline__ V3<double> fb_direction(V3<double> p, V3<double> closest, V3<double> face_normal) {
  const V3<double> d = p - closest;
  const double norm = sqrt(dot(d, d));
  return norm > 1.0e-12 ? v3<double>(d.x / norm, d.y / norm, d.z / norm) : face_normal;
}

// Step start, phase 1 (begin_contact_step / begin_mesh_step, contact.py:171-239):
// one warp per registered vertex.
__device__ inline void fb_begin_frames(const StepArgs& a, const Team team) {
  const FrictionArgs& f = a.fc;
  const int lane = threadIdx.x & 31;
  const int warps = team.size * kWarps;
  for (int c = team.rank * kWarps + (threadIdx.x >> 5); c < f.count; c += warps) {
    const int node = f.nodes[c];
    const V3<double> p = load3d(a.position, node);
    V3<double> n, t1, t2;
    int candidate = 1;
    if (f.kind == kBoundaryMesh) {
      V3<double> closest, face_normal;
      double dist2;
      fb_mesh_closest(f, p, node, a.position, closest, face_normal, dist2);
      candidate = sqrt(dist2) - f.radius <= 5.0 * f.radius;
      n = fb_direction(p, closest, face_normal);
      // Gram-Schmidt from the axis least parallel to n (first on ties).
      int axis = 0;
      for (int d = 1; d < 3; ++d)
        if (fabs(n[d]) < fabs(n[axis])) axis = d;
      V3<double> unit = v3<double>(0.0, 0.0, 0.0);
      unit[axis] = 1.0;
      t1 = unit - dot(n, unit) * n;
      const double t1_norm = sqrt(dot(t1, t1));
      t1 = v3<double>(t1.x / t1_norm, t1.y / t1_norm, t1.z / t1_norm);
    } else {
      n = fb_normal(f, p);
      // GetLocalFrame: t1 = normalize(n x e_i) for the axis maximising |n x e_i|.
      V3<double> best = v3<double>(0.0, 0.0, 0.0);
      for (int i = 0; i < 3; ++i) {
        V3<double> axis = v3<double>(0.0, 0.0, 0.0);
        axis[i] = 1.0;
        const V3<double> candidate_axis = cross(n, axis);
        if (dot(candidate_axis, candidate_axis) > dot(best, best)) best = candidate_axis;
      }
      const double best_norm = sqrt(dot(best, best));
      t1 = v3<double>(best.x / best_norm, best.y / best_norm, best.z / best_norm);
    }
    t2 = cross(n, t1);
    const double t2_norm = sqrt(dot(t2, t2));
    t2 = v3<double>(t2.x / t2_norm, t2.y / t2_norm, t2.z / t2_norm);
    if (lane == 0) {
      store3(f.normal, c, n);
      store3(f.tangent1, c, t1);
      store3(f.tangent2, c, t2);
      f.candidate[c] = candidate;
      // A vertex outside the candidate list restarts its warm start at zero.
      if (!candidate) f.multiplier[c] = 0.0;
      f.lambda_t[2 * c] = f.lambda_t[2 * c + 1] = 0.0;
    }
  }
}

// Step start, phase 2 (contact_delassus, contact.py:242-256): W and r, one thread per entry.
__device__ inline void fb_begin_delassus(const StepArgs& a, const Team team) {
  const FrictionArgs& f = a.fc;
  const int k = f.count;
  const long long entries = static_cast<long long>(k) * k;
  const long long threads = static_cast<long long>(team.size) * blockDim.x;
  for (long long t = static_cast<long long>(team.rank) * blockDim.x + threadIdx.x; t < entries; t += threads) {
    const int i = static_cast<int>(t / k), j = static_cast<int>(t % k);
    const int low = min(i, j), high = max(i, j);
    const double w = dot(load3d(f.normal, low), load3d(f.normal, high)) * f.block[static_cast<long long>(high) * k + low];
    f.delassus[t] = w;
    if (i == j) f.regularization[i] = fmax(a.dt * a.dt * w, 1.0e-10);
  }
}

// omega, E and phi of the Fischer-Burmeister function (contact.py:150-156).
__device__ __forceinline__ void fb_complementarity(double delta, double lam, double r, double& omega, double& e,
                                                   double& phi) {
  double s = sqrt(delta * delta + r * r * lam * lam);
  if (s < 1.0e-14) s = 1.0e-14;
  omega = 1.0 - delta / s;
  e = (1.0 - r * lam / s) * r;
  phi = delta + r * lam - s;
}

// Per-contact force omega lambda n (+ lambda_t . t) (contact_forces, contact.py:376-392).
__device__ __forceinline__ void fb_forces(const FrictionArgs& f, bool tangential) {
  for (int c = threadIdx.x; c < f.count; c += blockDim.x) {
    const double scale = f.omega[c] * f.multiplier[c];
    V3<double> value = scale * load3d(f.normal, c);
    if (tangential)
      value = value + f.lambda_t[2 * c] * load3d(f.tangent1, c) + f.lambda_t[2 * c + 1] * load3d(f.tangent2, c);
    store3(f.force, c, value);
  }
}

// response_c = sum_k B[c][order_k] f_order_k over the coupled candidates
// (contact_response, contact.py:395-409): one warp per contact, fixed-order sum.
__device__ inline void fb_response(const FrictionArgs& f, int active) {
  const int lane = threadIdx.x & 31;
  for (int c = threadIdx.x >> 5; c < f.count; c += kWarps) {
    const double* row = f.block + static_cast<long long>(c) * f.count;
    double rx = 0.0, ry = 0.0, rz = 0.0;
    for (int k = lane; k < active; k += 32) {
      const int j = f.order[k];
      const double b = row[j];
      rx += b * f.force[3 * j];
      ry += b * f.force[3 * j + 1];
      rz += b * f.force[3 * j + 2];
    }
    rx = warp_sum(rx);
    ry = warp_sum(ry);
    rz = warp_sum(rz);
    if (lane == 0) store3(f.response, c, v3<double>(rx, ry, rz));
  }
}

// Solves M[:n,:n] x = rhs[:n] in place with Eigen's LDL^T (left-looking,
// pivoting on the largest remaining diagonal entry, pseudo-inverse of D) as
// the reference's ldlt_solve (dense.py:40-106), by one block: the pivot search
// is a block reduction, each column update one warp per row.
__device__ inline void fb_ldlt_solve(double* m, int ld, int n, double* rhs, int* permutation, double* work) {
  __shared__ double s_value[kWarps];
  __shared__ int s_index[kWarps];
  __shared__ int s_pivot;
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  auto at = [&](int i, int j) -> double& { return m[static_cast<long long>(i) * ld + j]; };
  for (int i = threadIdx.x; i < n; i += blockDim.x) permutation[i] = i;
  for (int k = 0; k < n; ++k) {
    // First index of the largest |M_ii|, i >= k.
    double best = -1.0;
    int index = n;
    for (int i = k + threadIdx.x; i < n; i += blockDim.x) {
      const double v = fabs(at(i, i));
      if (v > best) {
        best = v;
        index = i;
      }
    }
#pragma unroll
    for (int offset = 16; offset > 0; offset >>= 1) {
      const double other = __shfl_xor_sync(0xffffffffu, best, offset);
      const int other_index = __shfl_xor_sync(0xffffffffu, index, offset);
      if (other > best || (other == best && other_index < index)) {
        best = other;
        index = other_index;
      }
    }
    if (lane == 0) {
      s_value[warp] = best;
      s_index[warp] = index;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      double v = s_value[0];
      int b = s_index[0];
      for (int w = 1; w < kWarps; ++w) {
        if (s_value[w] > v || (s_value[w] == v && s_index[w] < b)) {
          v = s_value[w];
          b = s_index[w];
        }
      }
      s_pivot = b < n ? b : k;
    }
    __syncthreads();
    const int biggest = s_pivot;
    if (biggest != k) {
      // Eigen's symmetric transposition restricted to the lower triangle; the
      // three loops touch disjoint entries.
      for (int j = threadIdx.x; j < k; j += blockDim.x) {
        const double t = at(k, j);
        at(k, j) = at(biggest, j);
        at(biggest, j) = t;
      }
      for (int i = biggest + 1 + threadIdx.x; i < n; i += blockDim.x) {
        const double t = at(i, k);
        at(i, k) = at(i, biggest);
        at(i, biggest) = t;
      }
      for (int i = k + 1 + threadIdx.x; i < biggest; i += blockDim.x) {
        const double t = at(i, k);
        at(i, k) = at(biggest, i);
        at(biggest, i) = t;
      }
      if (threadIdx.x == 0) {
        const double t = at(k, k);
        at(k, k) = at(biggest, biggest);
        at(biggest, biggest) = t;
        const int p = permutation[k];
        permutation[k] = permutation[biggest];
        permutation[biggest] = p;
      }
      __syncthreads();
    }
    if (warp == 0) {
      double sum = 0.0;
      for (int j = lane; j < k; j += 32) sum += at(k, j) * at(k, j) * at(j, j);
      sum = warp_sum(sum);
      if (lane == 0) at(k, k) = at(k, k) - sum;
    }
    __syncthreads();
    const double pivot = at(k, k);
    for (int i = k + 1 + warp; i < n; i += kWarps) {
      double sum = 0.0;
      for (int j = lane; j < k; j += 32) sum += at(i, j) * at(j, j) * at(k, j);
      sum = warp_sum(sum);
      if (lane == 0) {
        double v = at(i, k) - sum;
        if (pivot != 0.0) v = v / pivot;
        at(i, k) = v;
      }
    }
    __syncthreads();
  }
  // L z = P rhs, D y = z (pseudo-inverse), L^T w = y, rhs = P^T w.
  if (warp == 0) {
    for (int i = 0; i < n; ++i) {
      double sum = 0.0;
      for (int j = lane; j < i; j += 32) sum += at(i, j) * work[j];
      sum = warp_sum(sum);
      if (lane == 0) work[i] = rhs[permutation[i]] - sum;
      __syncwarp();
    }
    for (int i = lane; i < n; i += 32) {
      const double d = at(i, i);
      work[i] = fabs(d) > DBL_MIN ? work[i] / d : 0.0;
    }
    __syncwarp();
    for (int i = n - 1; i >= 0; --i) {
      double sum = 0.0;
      for (int j = i + 1 + lane; j < n; j += 32) sum += at(j, i) * work[j];
      sum = warp_sum(sum);
      if (lane == 0) work[i] = work[i] - sum;
      __syncwarp();
    }
  }
  __syncthreads();
  for (int i = threadIdx.x; i < n; i += blockDim.x) rhs[permutation[i]] = work[i];
  __syncthreads();
}

// One iteration's contact section by one block (FrictionalContact.iterate,
// contact.py:909-984): scalars at the iterate, compaction of the coupled
// candidates, one Newton step on lambda, the Coulomb update and the final
// forces. The caller's barrier publishes the forces and the order to the team.
__device__ inline void fb_newton(const StepArgs& a) {
  const FrictionArgs& f = a.fc;
  const int k_count = f.count;
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  __shared__ int s_warp_count[kWarps];
  __shared__ int s_base;
  // Scalars (contact_scalars / mesh_contact_scalars, contact.py:259-373), one warp per contact.
  for (int c = warp; c < k_count; c += kWarps) {
    const int node = f.nodes[c];
    double delta = 0.0, omega = 0.0, e = 1.0, phi = 0.0;
    if (f.candidate[c] != 0) {
      const V3<double> p = load3d(a.prev, node);
      if (f.kind == kBoundaryMesh) {
        V3<double> closest, face_normal;
        double dist2;
        fb_mesh_closest(f, p, node, a.prev, closest, face_normal, dist2);
        delta = dot(p - closest, load3d(f.normal, c)) - f.radius;
      } else {
        delta = fb_gap(f, p);
      }
      fb_complementarity(delta, f.multiplier[c], f.regularization[c], omega, e, phi);
    }
    if (lane == 0) {
      f.omega[c] = omega;
      f.diagonal[c] = e;
      f.residual[c] = phi;
    }
  }
  // Compaction of omega != 0 in candidate order (contact_active_scan, contact.py:476-499).
  if (threadIdx.x == 0) s_base = 0;
  __syncthreads();
  for (int start = 0; start < k_count; start += blockDim.x) {
    const int c = start + threadIdx.x;
    const bool flag = c < k_count && f.omega[c] != 0.0;
    const unsigned ballot = __ballot_sync(0xffffffffu, flag);
    if (lane == 0) s_warp_count[warp] = __popc(ballot);
    __syncthreads();
    int offset = s_base;
    for (int w = 0; w < warp; ++w) offset += s_warp_count[w];
    offset += __popc(ballot & ((1u << lane) - 1u));
    if (c < k_count) {
      f.slot[c] = flag ? offset : -1;
      if (flag) f.order[offset] = c;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      int total = 0;
      for (int w = 0; w < kWarps; ++w) total += s_warp_count[w];
      s_base += total;
    }
    __syncthreads();
  }
  const int active = s_base;
  if (threadIdx.x == 0) *f.active = active;
  // Newton right-hand side with the current forces (contact.py:430-447).
  fb_forces(f, true);
  __syncthreads();
  fb_response(f, active);
  __syncthreads();
  for (int c = threadIdx.x; c < k_count; c += blockDim.x) {
    const int node = f.nodes[c];
    const V3<double> n = load3d(f.normal, c);
    const V3<double> point = load3d(a.prev, node);
    const V3<double> solved = v3<double>(fb_solved(a, node, 0), fb_solved(a, node, 1), fb_solved(a, node, 2));
    f.rhs[c] = -f.residual[c] + f.omega[c] * dot(n, point) - f.omega[c] * dot(n, solved + load3d(f.response, c));
  }
  __syncthreads();
  // Coupled block Omega W Omega + E (contact_system, contact.py:502-528) and its solve.
  for (long long t = threadIdx.x; t < static_cast<long long>(active) * active; t += blockDim.x) {
    const int i = static_cast<int>(t / active), j = static_cast<int>(t % active);
    const int p = f.order[i], q = f.order[j];
    double value = f.omega[p] * f.delassus[static_cast<long long>(p) * k_count + q] * f.omega[q];
    if (i == j) value += f.diagonal[p];
    f.matrix[static_cast<long long>(i) * k_count + j] = value;
    if (j == 0) f.compact[i] = f.rhs[p];
  }
  __syncthreads();
  if (active > 0) fb_ldlt_solve(f.matrix, k_count, active, f.compact, f.permutation, f.work);
  // lambda <- clamp(lambda + d lambda, 0, 1e8) (contact_update, contact.py:531-546).
  for (int c = threadIdx.x; c < k_count; c += blockDim.x) {
    const int slot = f.slot[c];
    const double step = slot >= 0 ? f.compact[slot] : f.rhs[c] / f.diagonal[c];
    f.multiplier[c] = fmin(fmax(f.multiplier[c] + step, 0.0), 1.0e8);
  }
  __syncthreads();
  if (f.friction > 0.0) {
    // Stick/slip projection with the normal-only response (contact_friction, contact.py:549-592).
    fb_forces(f, false);
    __syncthreads();
    fb_response(f, active);
    __syncthreads();
    for (int c = threadIdx.x; c < k_count; c += blockDim.x) {
      if (f.multiplier[c] <= 0.0) {
        f.lambda_t[2 * c] = f.lambda_t[2 * c + 1] = 0.0;
        continue;
      }
      const int node = f.nodes[c];
      const V3<double> solved = v3<double>(fb_solved(a, node, 0), fb_solved(a, node, 1), fb_solved(a, node, 2));
      const V3<double> step = solved + load3d(f.response, c) - load3d(a.position, node);
      const V3<double> n = load3d(f.normal, c), t1 = load3d(f.tangent1, c), t2 = load3d(f.tangent2, c);
      const V3<double> tangential = step - dot(step, n) * n;
      const double u1 = dot(tangential, t1), u2 = dot(tangential, t2);
      const double diagonal = f.block[static_cast<long long>(c) * k_count + c];
      const double w11 = dot(t1, t1) * diagonal, w12 = dot(t1, t2) * diagonal, w22 = dot(t2, t2) * diagonal;
      const double determinant = w11 * w22 - w12 * w12;
      double s1 = 0.0, s2 = 0.0;
      if (fabs(determinant) > 1.0e-20) {
        s1 = -(w22 * u1 - w12 * u2) / determinant;
        s2 = -(-w12 * u1 + w11 * u2) / determinant;
      }
      const double radius = f.friction * f.multiplier[c];
      if (sqrt(s1 * s1 + s2 * s2) <= radius + 1.0e-14) {
        f.lambda_t[2 * c] = s1;
        f.lambda_t[2 * c + 1] = s2;
      } else {
        const double magnitude = sqrt(u1 * u1 + u2 * u2);
        f.lambda_t[2 * c] = magnitude > 1.0e-14 ? -radius * u1 / magnitude : 0.0;
        f.lambda_t[2 * c + 1] = magnitude > 1.0e-14 ? -radius * u2 / magnitude : 0.0;
      }
    }
    __syncthreads();
  }
  fb_forces(f, true);
}

// ---------------------------------------------------------------------------
// The same Newton step spread over the whole team, for large contact sets
// (more than kTeamContacts registered vertices): every per-contact and
// per-entry loop is distributed over the team's blocks, and the coupled
// block, symmetric positive definite (contact.py:33-39), is factorised by a
// right-looking Cholesky in 32-wide panels: one warp factors the diagonal
// tile in shared memory, the team solves the panel below (a warp per row)
// and updates the trailing lower triangle (a thread per entry), with a team
// barrier between the three.

constexpr int kTeamContacts = 32;
constexpr int kPanel = 32;

__device__ __forceinline__ int team_warp(const Team team) { return team.rank * kWarps + (threadIdx.x >> 5); }

// Scalars at the iterate, one warp per contact over the team.
__device__ inline void fb_scalars_team(const StepArgs& a, const Team team) {
  const FrictionArgs& f = a.fc;
  const int lane = threadIdx.x & 31;
  for (int c = team_warp(team); c < f.count; c += team.size * kWarps) {
    const int node = f.nodes[c];
    double delta = 0.0, omega = 0.0, e = 1.0, phi = 0.0;
    if (f.candidate[c] != 0) {
      const V3<double> p = load3d(a.prev, node);
      if (f.kind == kBoundaryMesh) {
        V3<double> closest, face_normal;
        double dist2;
        fb_mesh_closest(f, p, node, a.prev, closest, face_normal, dist2);
        delta = dot(p - closest, load3d(f.normal, c)) - f.radius;
      } else {
        delta = fb_gap(f, p);
      }
      fb_complementarity(delta, f.multiplier[c], f.regularization[c], omega, e, phi);
    }
    if (lane == 0) {
      f.omega[c] = omega;
      f.diagonal[c] = e;
      f.residual[c] = phi;
    }
  }
}

// Ordered compaction of omega != 0 and the current forces, by one block.
__device__ inline void fb_compact_block(const FrictionArgs& f) {
  __shared__ int s_warp_count[kWarps];
  __shared__ int s_base;
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  if (threadIdx.x == 0) s_base = 0;
  __syncthreads();
  for (int start = 0; start < f.count; start += blockDim.x) {
    const int c = start + threadIdx.x;
    const bool flag = c < f.count && f.omega[c] != 0.0;
    const unsigned ballot = __ballot_sync(0xffffffffu, flag);
    if (lane == 0) s_warp_count[warp] = __popc(ballot);
    __syncthreads();
    int offset = s_base;
    for (int w = 0; w < warp; ++w) offset += s_warp_count[w];
    offset += __popc(ballot & ((1u << lane) - 1u));
    if (c < f.count) {
      f.slot[c] = flag ? offset : -1;
      if (flag) f.order[offset] = c;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      int total = 0;
      for (int w = 0; w < kWarps; ++w) total += s_warp_count[w];
      s_base += total;
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) *f.active = s_base;
  fb_forces(f, true);
}

__device__ inline void fb_forces_team(const FrictionArgs& f, const Team team, bool tangential) {
  for (int c = team.rank * blockDim.x + threadIdx.x; c < f.count; c += team.size * blockDim.x) {
    const double scale = f.omega[c] * f.multiplier[c];
    V3<double> value = scale * load3d(f.normal, c);
    if (tangential)
      value = value + f.lambda_t[2 * c] * load3d(f.tangent1, c) + f.lambda_t[2 * c + 1] * load3d(f.tangent2, c);
    store3(f.force, c, value);
  }
}

__device__ inline void fb_response_team(const FrictionArgs& f, const Team team, int active) {
  const int lane = threadIdx.x & 31;
  for (int c = team_warp(team); c < f.count; c += team.size * kWarps) {
    const double* row = f.block + static_cast<long long>(c) * f.count;
    double rx = 0.0, ry = 0.0, rz = 0.0;
#pragma unroll 4
    for (int k = lane; k < active; k += 32) {
      const int j = f.order[k];
      const double b = row[j];
      rx += b * f.force[3 * j];
      ry += b * f.force[3 * j + 1];
      rz += b * f.force[3 * j + 2];
    }
    rx = warp_sum(rx);
    ry = warp_sum(ry);
    rz = warp_sum(rz);
    if (lane == 0) store3(f.response, c, v3<double>(rx, ry, rz));
  }
}

// The response of every contact and, by the same warp, its right-hand side
// (contact_newton_rhs, contact.py:430-447).
__device__ inline void fb_response_rhs_team(const StepArgs& a, const Team team, int active) {
  const FrictionArgs& f = a.fc;
  const int lane = threadIdx.x & 31;
  for (int c = team_warp(team); c < f.count; c += team.size * kWarps) {
    const double* row = f.block + static_cast<long long>(c) * f.count;
    double rx = 0.0, ry = 0.0, rz = 0.0;
#pragma unroll 4
    for (int k = lane; k < active; k += 32) {
      const int j = f.order[k];
      const double b = row[j];
      rx += b * f.force[3 * j];
      ry += b * f.force[3 * j + 1];
      rz += b * f.force[3 * j + 2];
    }
    rx = warp_sum(rx);
    ry = warp_sum(ry);
    rz = warp_sum(rz);
    if (lane == 0) {
      const V3<double> response = v3<double>(rx, ry, rz);
      store3(f.response, c, response);
      const int node = f.nodes[c];
      const V3<double> n = load3d(f.normal, c);
      const V3<double> point = load3d(a.prev, node);
      const V3<double> solved = v3<double>(fb_solved(a, node, 0), fb_solved(a, node, 1), fb_solved(a, node, 2));
      f.rhs[c] = -f.residual[c] + f.omega[c] * dot(n, point) - f.omega[c] * dot(n, solved + response);
    }
  }
}

// The lower triangle of the coupled block Omega W Omega + E (contact_system, contact.py:502-528).
__device__ inline void fb_matrix_team(const FrictionArgs& f, const Team team, int active) {
  const long long entries = static_cast<long long>(active) * active;
  for (long long t = static_cast<long long>(team.rank) * blockDim.x + threadIdx.x; t < entries;
       t += static_cast<long long>(team.size) * blockDim.x) {
    const int i = static_cast<int>(t / active), j = static_cast<int>(t % active);
    if (j > i) continue;
    const int p = f.order[i], q = f.order[j];
    double value = f.omega[p] * f.delassus[static_cast<long long>(p) * f.count + q] * f.omega[q];
    if (i == j) value += f.diagonal[p];
    f.matrix[static_cast<long long>(i) * f.count + j] = value;
  }
}

// In-place Cholesky of the lower triangle of m[:n, :n] (leading dimension
// ld) by the team. Returns false when a team barrier gave up. Two team
// barriers per panel: the first block folds the next diagonal tile's
// trailing update into its own share and factors that tile right away.
__device__ inline bool fb_cholesky_team(const StepArgs& a, const Team team, double* m, int ld, int n,
                                        double* tile /* shared [kPanel * (kPanel + 1)] */) {
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  auto at = [&](int i, int j) -> double& { return m[static_cast<long long>(i) * ld + j]; };
  // Diagonal tile at c0 (w rows) by warp 0 of the calling block: lane r owns row r.
  auto factor_tile = [&](int c0, int w) {
    if (warp != 0) return;
    for (int r = 0; r < w; ++r)
      if (lane <= r) tile[r * (kPanel + 1) + lane] = at(c0 + r, c0 + lane);
    __syncwarp();
    for (int k = 0; k < w; ++k) {
      double d = tile[k * (kPanel + 1) + k];
      d = d > 0.0 ? sqrt(d) : sqrt(DBL_MIN);
      __syncwarp();
      if (lane == k) tile[k * (kPanel + 1) + k] = d;
      if (lane > k && lane < w) tile[lane * (kPanel + 1) + k] /= d;
      __syncwarp();
      if (lane > k && lane < w) {
        const double lk = tile[lane * (kPanel + 1) + k];
        for (int c = k + 1; c <= lane; ++c) tile[lane * (kPanel + 1) + c] -= lk * tile[c * (kPanel + 1) + k];
      }
      __syncwarp();
    }
    for (int r = 0; r < w; ++r)
      if (lane <= r) at(c0 + r, c0 + lane) = tile[r * (kPanel + 1) + lane];
  };
  if (team.rank == 0) factor_tile(0, min(kPanel, n));
  if (!grid_sync(a.barrier, a.status, team.size, team.rank)) return false;
  for (int c0 = 0; c0 + kPanel < n; c0 += kPanel) {
    const int w = kPanel;
    const int t0 = c0 + w, w2 = min(kPanel, n - t0);
    // Panel below: L_ip = M_ip L_pp^-T, a warp per row.
    for (int r = threadIdx.x; r < w * w; r += blockDim.x) {
      const int i = r / w, j = r % w;
      if (j <= i) tile[i * (kPanel + 1) + j] = at(c0 + i, c0 + j);
    }
    __syncthreads();
    for (int row = t0 + team_warp(team); row < n; row += team.size * kWarps) {
      double v = lane < w ? at(row, c0 + lane) : 0.0;
      for (int j = 0; j < w; ++j) {
        const double x = __shfl_sync(0xffffffffu, v, j) / tile[j * (kPanel + 1) + j];
        if (lane == j) v = x;
        if (lane > j && lane < w) v -= x * tile[lane * (kPanel + 1) + j];
      }
      if (lane < w) at(row, c0 + lane) = v;
    }
    if (!grid_sync(a.barrier, a.status, team.size, team.rank)) return false;
    // Trailing lower triangle M_ij -= L_ip . L_jp; the next diagonal tile
    // (rows below t0 + w2) by the first block, which then factors it.
    auto update = [&](int i, int j) {
      const double* li = m + static_cast<long long>(i) * ld + c0;
      const double* lj = m + static_cast<long long>(j) * ld + c0;
      double sum = 0.0;
#pragma unroll 8
      for (int l = 0; l < w; ++l) sum += li[l] * lj[l];
      at(i, j) -= sum;
    };
    const int rest = n - t0;
    const long long entries = static_cast<long long>(rest) * rest;
    for (long long t = static_cast<long long>(team.rank) * blockDim.x + threadIdx.x; t < entries;
         t += static_cast<long long>(team.size) * blockDim.x) {
      const int i = t0 + static_cast<int>(t / rest), j = t0 + static_cast<int>(t % rest);
      if (j > i || i < t0 + w2) continue;
      update(i, j);
    }
    if (team.rank == 0) {
      for (int t = threadIdx.x; t < w2 * w2; t += blockDim.x) {
        const int i = t0 + t / w2, j = t0 + t % w2;
        if (j <= i) update(i, j);
      }
      __syncthreads();
      factor_tile(t0, w2);
    }
    if (!grid_sync(a.barrier, a.status, team.size, team.rank)) return false;
  }
  return true;
}

// L L^T x = rhs on the factor from fb_cholesky_team, by one block: panel by
// panel, the off-panel part by a warp per row, the tile by warp 0.
__device__ inline void fb_cholesky_solve_block(const double* m, int ld, int n, double* x,
                                               double* tile /* shared [kPanel * (kPanel + 1)] */) {
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  auto at = [&](int i, int j) -> double { return m[static_cast<long long>(i) * ld + j]; };
  auto load_tile = [&](int c0, int w) {
    for (int r = threadIdx.x; r < w * w; r += blockDim.x) {
      const int i = r / w, j = r % w;
      if (j <= i) tile[i * (kPanel + 1) + j] = at(c0 + i, c0 + j);
    }
  };
  for (int c0 = 0; c0 < n; c0 += kPanel) {
    const int w = min(kPanel, n - c0);
    load_tile(c0, w);
    for (int r = c0 + warp; r < c0 + w; r += kWarps) {
      double sum = 0.0;
      for (int c = lane; c < c0; c += 32) sum += at(r, c) * x[c];
      sum = warp_sum(sum);
      if (lane == 0) x[r] -= sum;
    }
    __syncthreads();
    if (warp == 0) {
      double v = lane < w ? x[c0 + lane] : 0.0;
      for (int j = 0; j < w; ++j) {
        const double y = __shfl_sync(0xffffffffu, v, j) / tile[j * (kPanel + 1) + j];
        if (lane == j) v = y;
        if (lane > j && lane < w) v -= y * tile[lane * (kPanel + 1) + j];
      }
      if (lane < w) x[c0 + lane] = v;
    }
    __syncthreads();
  }
  for (int c0 = ((n - 1) / kPanel) * kPanel; c0 >= 0; c0 -= kPanel) {
    const int w = min(kPanel, n - c0);
    load_tile(c0, w);
    for (int r = c0 + warp; r < c0 + w; r += kWarps) {
      double sum = 0.0;
      for (int c = c0 + w + lane; c < n; c += 32) sum += at(c, r) * x[c];
      sum = warp_sum(sum);
      if (lane == 0) x[r] -= sum;
    }
    __syncthreads();
    if (warp == 0) {
      double v = lane < w ? x[c0 + lane] : 0.0;
      for (int j = w - 1; j >= 0; --j) {
        const double y = __shfl_sync(0xffffffffu, v, j) / tile[j * (kPanel + 1) + j];
        if (lane == j) v = y;
        if (lane < j) v -= y * tile[j * (kPanel + 1) + lane];
      }
      if (lane < w) x[c0 + lane] = v;
    }
    __syncthreads();
  }
}

// Multiplier update (contact_update, contact.py:531-546) and the contact's
// force right after it: normal only when friction follows, else final.
__device__ inline void fb_update_team(const FrictionArgs& f, const Team team) {
  const bool tangential = !(f.friction > 0.0);
  for (int c = team.rank * blockDim.x + threadIdx.x; c < f.count; c += team.size * blockDim.x) {
    const int slot = f.slot[c];
    const double step = slot >= 0 ? f.compact[slot] : f.rhs[c] / f.diagonal[c];
    const double lambda = fmin(fmax(f.multiplier[c] + step, 0.0), 1.0e8);
    f.multiplier[c] = lambda;
    V3<double> value = (f.omega[c] * lambda) * load3d(f.normal, c);
    if (tangential)
      value = value + f.lambda_t[2 * c] * load3d(f.tangent1, c) + f.lambda_t[2 * c + 1] * load3d(f.tangent2, c);
    store3(f.force, c, value);
  }
}

__device__ inline void fb_friction_team(const StepArgs& a, const Team team) {
  const FrictionArgs& f = a.fc;
  for (int c = team.rank * blockDim.x + threadIdx.x; c < f.count; c += team.size * blockDim.x) {
    if (f.multiplier[c] <= 0.0) {
      f.lambda_t[2 * c] = f.lambda_t[2 * c + 1] = 0.0;
      continue;
    }
    const int node = f.nodes[c];
    const V3<double> solved = v3<double>(fb_solved(a, node, 0), fb_solved(a, node, 1), fb_solved(a, node, 2));
    const V3<double> step = solved + load3d(f.response, c) - load3d(a.position, node);
    const V3<double> n = load3d(f.normal, c), t1 = load3d(f.tangent1, c), t2 = load3d(f.tangent2, c);
    const V3<double> tangential = step - dot(step, n) * n;
    const double u1 = dot(tangential, t1), u2 = dot(tangential, t2);
    const double diagonal = f.block[static_cast<long long>(c) * f.count + c];
    const double w11 = dot(t1, t1) * diagonal, w12 = dot(t1, t2) * diagonal, w22 = dot(t2, t2) * diagonal;
    const double determinant = w11 * w22 - w12 * w12;
    double s1 = 0.0, s2 = 0.0;
    if (fabs(determinant) > 1.0e-20) {
      s1 = -(w22 * u1 - w12 * u2) / determinant;
      s2 = -(-w12 * u1 + w11 * u2) / determinant;
    }
    const double radius = f.friction * f.multiplier[c];
    if (sqrt(s1 * s1 + s2 * s2) <= radius + 1.0e-14) {
      f.lambda_t[2 * c] = s1;
      f.lambda_t[2 * c + 1] = s2;
    } else {
      const double magnitude = sqrt(u1 * u1 + u2 * u2);
      f.lambda_t[2 * c] = magnitude > 1.0e-14 ? -radius * u1 / magnitude : 0.0;
      f.lambda_t[2 * c + 1] = magnitude > 1.0e-14 ? -radius * u2 / magnitude : 0.0;
    }
  }
}

// The whole contact section of one iteration for large contact sets; every
// block of the team calls it after A^{-1} b is complete. Returns false when a
// team barrier gave up.
__device__ inline bool fb_newton_team(const StepArgs& a, const Team team) {
  __shared__ double tile[kPanel * (kPanel + 1)];
  const FrictionArgs& f = a.fc;
  fb_scalars_team(a, team);
  if (!grid_sync(a.barrier, a.status, team.size, team.rank)) return false;
  if (team.rank == 0) fb_compact_block(f);
  if (!grid_sync(a.barrier, a.status, team.size, team.rank)) return false;
  const int active = *reinterpret_cast<volatile int*>(f.active);
  fb_response_rhs_team(a, team, active);
  fb_matrix_team(f, team, active);
  if (!grid_sync(a.barrier, a.status, team.size, team.rank)) return false;
  if (active > 0) {
    if (!fb_cholesky_team(a, team, f.matrix, f.count, active, tile)) return false;
    if (team.rank == 0) {
      for (int i = threadIdx.x; i < active; i += blockDim.x) f.compact[i] = f.rhs[f.order[i]];
      __syncthreads();
      fb_cholesky_solve_block(f.matrix, f.count, active, f.compact, tile);
    }
    if (!grid_sync(a.barrier, a.status, team.size, team.rank)) return false;
  }
  fb_update_team(f, team);
  if (!grid_sync(a.barrier, a.status, team.size, team.rank)) return false;
  if (f.friction > 0.0) {
    fb_response_team(f, team, active);
    if (!grid_sync(a.barrier, a.status, team.size, team.rank)) return false;
    fb_friction_team(a, team);
    fb_forces_team(f, team, true);
    if (!grid_sync(a.barrier, a.status, team.size, team.rank)) return false;
  }
  return true;
}

// x_i += sum_k P[i][order_k] f_order_k (contact_solution, contact.py:412-427).
__device__ __forceinline__ V3<double> fb_correction(const FrictionArgs& f, int i, int active) {
  const double* row = f.panel + static_cast<long long>(i) * f.count;
  V3<double> value = v3<double>(0.0, 0.0, 0.0);
  for (int k = 0; k < active; ++k) {
    const int j = f.order[k];
    value = value + row[j] * load3d(f.force, j);
  }
  return value;
}

// Post-solve restitution (apply_restitution / apply_mesh_restitution,
// contact.py:595-667), one warp per contact.
__device__ inline void fb_restitution(const StepArgs& a, const Team team) {
  const FrictionArgs& f = a.fc;
  const int lane = threadIdx.x & 31;
  const int warps = team.size * kWarps;
  for (int c = team.rank * kWarps + (threadIdx.x >> 5); c < f.count; c += warps) {
    if (f.multiplier[c] <= 0.0) continue;
    const int node = f.nodes[c];
    const V3<double> point = load3d(a.x, node);
    double distance, slop;
    V3<double> n;
    if (f.kind == kBoundaryMesh) {
      V3<double> closest, face_normal;
      double dist2;
      fb_mesh_closest(f, point, node, f.surface, closest, face_normal, dist2);
      const V3<double> reference = load3d(f.normal, c);
      distance = dot(point - closest, reference) - f.radius;
      n = fb_direction(point, closest, face_normal);
      if (dot(n, reference) < 0.0) n = v3<double>(-n.x, -n.y, -n.z);
      slop = 0.1 * f.radius;
    } else {
      distance = fb_gap(f, point);
      n = fb_normal(f, point);
      slop = 1.0e-8;
    }
    const double norm = sqrt(dot(n, n));
    if (norm <= 1.0e-12) continue;
    n = v3<double>(n.x / norm, n.y / norm, n.z / norm);
    if (distance > slop) continue;
    const double incoming = dot(load3d(a.velocity, node), n);
    if (incoming < 0.0) {
      const V3<double> moved = point - load3d(a.position, node);
      const double outgoing = dot(v3<double>(moved.x / a.dt, moved.y / a.dt, moved.z / a.dt), n);
      const double change = -f.restitution * incoming - outgoing;
      if (change > 0.0 && lane == 0) store3(a.x, node, point + (a.dt * change) * n);
    }
  }
}

}  // namespace pdb200
