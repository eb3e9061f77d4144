// The reference's mesh_contact state force (mesh_contact.py, the DiffPhD
// MeshContactStateForce): every surface vertex of body A against every face
// of body B with stiffness kn_left, and every surface vertex of B against
// every face of A with kn_right. Within `radius` of the closest point of a
// face, the vertex receives kn (radius - dist) n plus the friction
// -min(kf, mu fn / (|v_t| + eps)) v_t of its tangential velocity relative to
// the face; the face's corners receive the opposite force weighted by the
// closest point's barycentric coordinates. Evaluated once per step on the
// start-of-step state; the result enters the inertial target and carries no
// gradient (the reference's BackwardForce returns zero).
//
// Two passes with a fixed summation order: one thread per (vertex, face)
// pair writes that pair's force and weights; one thread per particle then
// sums, in order, its forces as a vertex of A, as a vertex of B, and the
// reactions as a corner of B's and of A's faces.
#include <cuda_runtime.h>

#include <cfloat>
#include <cmath>
#include <string>
#include <vector>

#include "../../include/pd_b200.h"
#include "pd_device.cuh"
#include "pd_geometry.cuh"
#include "solver_state.h"

namespace pdb200 {

namespace {

__device__ __forceinline__ V3<double> load_state3(const void* p, int f64, int i) {
  return v3<double>(state_load(p, f64, 3 * i), state_load(p, f64, 3 * i + 1), state_load(p, f64, 3 * i + 2));
}

// One thread per (vertex s, face f): force on the vertex and the closest point's weights.
__global__ void pair_forces_kernel(const void* q, const void* v, int f64, const int* vertices, int n_vertices,
                                   const int* faces, int n_faces, double radius, double kn, double kf, double mu,
                                   double* force, double* bary, int* pairs) {
  const long long t = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (t >= static_cast<long long>(n_vertices) * n_faces) return;
  const int s = static_cast<int>(t / n_faces);
  const int f = static_cast<int>(t % n_faces);
  double* out = force + 3 * t;
  double* weights_out = bary + 3 * t;
  for (int c = 0; c < 3; ++c) out[c] = weights_out[c] = 0.0;
  const int vid = vertices[s];
  const int i0 = faces[3 * f], i1 = faces[3 * f + 1], i2 = faces[3 * f + 2];
  const V3<double> p = load_state3(q, f64, vid);
  const V3<double> a = load_state3(q, f64, i0), b = load_state3(q, f64, i1), c = load_state3(q, f64, i2);
  const TrianglePoint closest = closest_point(p, a, b, c);
  const V3<double> d = p - closest.point;
  const double gap2 = dot3(d, d);
  if (gap2 >= radius * radius) return;
  const double gap = sqrt(gap2);
  V3<double> normal;
  if (gap > DBL_EPSILON) {
    normal = v3<double>(d.x / gap, d.y / gap, d.z / gap);
  } else {
    const V3<double> e1 = b - a, e2 = c - a;
    normal = v3<double>(e1.y * e2.z - e1.z * e2.y, e1.z * e2.x - e1.x * e2.z, e1.x * e2.y - e1.y * e2.x);
    const double length = sqrt(dot3(normal, normal));
    if (length <= DBL_EPSILON) return;
    normal = v3<double>(normal.x / length, normal.y / length, normal.z / length);
  }
  if (dot3(normal, d) < 0.0) normal = v3<double>(-normal.x, -normal.y, -normal.z);
  const double magnitude = kn * (radius - gap);
  const V3<double> w = closest.weights;
  const V3<double> face_velocity = w.x * load_state3(v, f64, i0) + w.y * load_state3(v, f64, i1) +
                                   w.z * load_state3(v, f64, i2);
  const V3<double> relative = load_state3(v, f64, vid) - face_velocity;
  const double along = dot3(relative, normal);
  const V3<double> tangential = v3<double>(relative.x - normal.x * along, relative.y - normal.y * along,
                                           relative.z - normal.z * along);
  const double speed = sqrt(dot3(tangential, tangential));
  V3<double> friction = v3<double>(0.0, 0.0, 0.0);
  if (speed > DBL_EPSILON) {
    const double coefficient = -fmin(kf, mu * magnitude / (speed + DBL_EPSILON));
    friction = v3<double>(coefficient * tangential.x, coefficient * tangential.y, coefficient * tangential.z);
  }
  out[0] = magnitude * normal.x + friction.x;
  out[1] = magnitude * normal.y + friction.y;
  out[2] = magnitude * normal.z + friction.z;
  weights_out[0] = w.x;
  weights_out[1] = w.y;
  weights_out[2] = w.z;
  atomicAdd(pairs, 1);
}

// One thread per particle: the fixed-order sum of its pair forces and reactions.
__global__ void gather_contact_kernel(int n, const int* slot_a, const int* slot_b, const double* force_ab,
                                      const double* bary_ab, int va, int fb, const double* force_ba,
                                      const double* bary_ba, int vb, int fa, const int* inc_a_off, const int* inc_a,
                                      const int* inc_b_off, const int* inc_b, double* out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double tx = 0.0, ty = 0.0, tz = 0.0;
  // As a vertex of A against the faces of B, and of B against the faces of A.
  if (slot_a[i] >= 0) {
    const double* row = force_ab + 3 * static_cast<size_t>(slot_a[i]) * fb;
    for (int f = 0; f < fb; ++f) {
      tx += row[3 * f];
      ty += row[3 * f + 1];
      tz += row[3 * f + 2];
    }
  }
  if (slot_b[i] >= 0) {
    const double* row = force_ba + 3 * static_cast<size_t>(slot_b[i]) * fa;
    for (int f = 0; f < fa; ++f) {
      tx += row[3 * f];
      ty += row[3 * f + 1];
      tz += row[3 * f + 2];
    }
  }
  // As a corner of a face of B pushed by A's vertices, then of A's faces by B's.
  for (int k = inc_b_off[i]; k < inc_b_off[i + 1]; ++k) {
    const int face = inc_b[2 * k], corner = inc_b[2 * k + 1];
    for (int s = 0; s < va; ++s) {
      const size_t pair = static_cast<size_t>(s) * fb + face;
      const double weight = bary_ab[3 * pair + corner];
      tx -= force_ab[3 * pair] * weight;
      ty -= force_ab[3 * pair + 1] * weight;
      tz -= force_ab[3 * pair + 2] * weight;
    }
  }
  for (int k = inc_a_off[i]; k < inc_a_off[i + 1]; ++k) {
    const int face = inc_a[2 * k], corner = inc_a[2 * k + 1];
    for (int s = 0; s < vb; ++s) {
      const size_t pair = static_cast<size_t>(s) * fa + face;
      const double weight = bary_ba[3 * pair + corner];
      tx -= force_ba[3 * pair] * weight;
      ty -= force_ba[3 * pair + 1] * weight;
      tz -= force_ba[3 * pair + 2] * weight;
    }
  }
  out[3 * i] = tx;
  out[3 * i + 1] = ty;
  out[3 * i + 2] = tz;
}

// Per particle, the (face, corner) entries of `faces` in face order (CSR).
void incidence(const std::vector<int32_t>& faces, int n, std::vector<int32_t>& offsets, std::vector<int32_t>& entries) {
  offsets.assign(n + 1, 0);
  for (int32_t node : faces) offsets[node + 1] += 1;
  for (int i = 0; i < n; ++i) offsets[i + 1] += offsets[i];
  entries.assign(2 * faces.size(), 0);
  std::vector<int32_t> fill(offsets.begin(), offsets.end() - 1);
  for (size_t f = 0; f < faces.size() / 3; ++f) {
    for (int corner = 0; corner < 3; ++corner) {
      const int32_t node = faces[3 * f + corner];
      const int32_t k = fill[node]++;
      entries[2 * k] = static_cast<int32_t>(f);
      entries[2 * k + 1] = corner;
    }
  }
}

}  // namespace

}  // namespace pdb200

int pd_evaluate_mesh_contact(PdSolver* s, const void* q, const void* v, int f64, cudaStream_t stream) {
  const double* p = s->mc_params;
  PD_CUDA(cudaMemsetAsync(s->mc_pairs.ptr, 0, sizeof(int), stream));
  const int threads = 256;
  struct Side {
    const DeviceBuffer& vertices;
    int count;
    const DeviceBuffer& faces;
    int face_count;
    double kn;
    DeviceBuffer& force;
    DeviceBuffer& bary;
  };
  const Side sides[2] = {{s->mc_vertices_a, s->mc_va, s->mc_faces_b, s->mc_fb, p[1], s->mc_force_ab, s->mc_bary_ab},
                         {s->mc_vertices_b, s->mc_vb, s->mc_faces_a, s->mc_fa, p[2], s->mc_force_ba, s->mc_bary_ba}};
  for (const Side& side : sides) {
    const long long pairs = static_cast<long long>(side.count) * side.face_count;
    const unsigned blocks = static_cast<unsigned>((pairs + threads - 1) / threads);
    pdb200::pair_forces_kernel<<<blocks, threads, 0, stream>>>(
        q, v, f64, side.vertices.as<int>(), side.count, side.faces.as<int>(), side.face_count, p[0], side.kn, p[3],
        p[4], side.force.as<double>(), side.bary.as<double>(), s->mc_pairs.as<int>());
  }
  pdb200::gather_contact_kernel<<<(s->n + threads - 1) / threads, threads, 0, stream>>>(
      s->n, s->mc_slot_a.as<int>(), s->mc_slot_b.as<int>(), s->mc_force_ab.as<double>(), s->mc_bary_ab.as<double>(),
      s->mc_va, s->mc_fb, s->mc_force_ba.as<double>(), s->mc_bary_ba.as<double>(), s->mc_vb, s->mc_fa,
      s->mc_inc_a_off.as<int>(), s->mc_inc_a.as<int>(), s->mc_inc_b_off.as<int>(), s->mc_inc_b.as<int>(),
      s->mc_force.as<double>());
  PD_CUDA(cudaGetLastError());
  return PD_OK;
}

extern "C" int pd_set_mesh_contact(PdSolver* s, double radius, double kn_left, double kn_right, double kf, double mu,
                                   int32_t n_faces_a, const int32_t* faces_a, int32_t n_faces_b,
                                   const int32_t* faces_b) {
  if (s == nullptr) return pd_set_error(PD_ERR_INVALID, "null solver");
  const char* names[5] = {"contact_radius", "kn_left", "kn_right", "kf", "mu"};
  const double values[5] = {radius, kn_left, kn_right, kf, mu};
  for (int k = 0; k < 5; ++k) {
    if (!std::isfinite(values[k]) || values[k] < 0.0)
      return pd_set_error(PD_ERR_INVALID, std::string("mesh_contact ") + names[k] + " must be finite and nonnegative");
  }
  if (n_faces_a <= 0 || n_faces_b <= 0 || faces_a == nullptr || faces_b == nullptr)
    return pd_set_error(PD_ERR_INVALID, "mesh_contact needs faces on both bodies");
  if (s->hex) return pd_set_error(PD_ERR_UNSUPPORTED, "Hex8 currently supports planar_energies, not frictional or mesh contact");
  std::vector<int32_t> fa(faces_a, faces_a + 3 * static_cast<size_t>(n_faces_a));
  std::vector<int32_t> fb(faces_b, faces_b + 3 * static_cast<size_t>(n_faces_b));
  for (const auto* faces : {&fa, &fb}) {
    for (int32_t node : *faces) {
      if (node < 0 || node >= s->n) return pd_set_error(PD_ERR_INVALID, "mesh_contact faces must reference existing particles");
    }
  }
  PD_CUDA(cudaSetDevice(s->device));
  // The sorted unique vertices of each body's faces and their slots.
  auto unique_vertices = [&](const std::vector<int32_t>& faces, std::vector<int32_t>& slot) {
    std::vector<char> used(s->n, 0);
    for (int32_t node : faces) used[node] = 1;
    std::vector<int32_t> list;
    slot.assign(s->n, -1);
    for (int i = 0; i < s->n; ++i) {
      if (used[i]) {
        slot[i] = static_cast<int32_t>(list.size());
        list.push_back(i);
      }
    }
    return list;
  };
  std::vector<int32_t> slot_a, slot_b;
  const std::vector<int32_t> vertices_a = unique_vertices(fa, slot_a);
  const std::vector<int32_t> vertices_b = unique_vertices(fb, slot_b);
  std::vector<int32_t> inc_a_off, inc_a, inc_b_off, inc_b;
  pdb200::incidence(fa, s->n, inc_a_off, inc_a);
  pdb200::incidence(fb, s->n, inc_b_off, inc_b);
  s->mc_va = static_cast<int>(vertices_a.size());
  s->mc_vb = static_cast<int>(vertices_b.size());
  s->mc_fa = n_faces_a;
  s->mc_fb = n_faces_b;
  for (int k = 0; k < 5; ++k) s->mc_params[k] = values[k];
  PD_CUDA(s->mc_vertices_a.upload(vertices_a));
  PD_CUDA(s->mc_vertices_b.upload(vertices_b));
  PD_CUDA(s->mc_faces_a.upload(fa));
  PD_CUDA(s->mc_faces_b.upload(fb));
  PD_CUDA(s->mc_slot_a.upload(slot_a));
  PD_CUDA(s->mc_slot_b.upload(slot_b));
  PD_CUDA(s->mc_inc_a_off.upload(inc_a_off));
  PD_CUDA(s->mc_inc_a.upload(inc_a));
  PD_CUDA(s->mc_inc_b_off.upload(inc_b_off));
  PD_CUDA(s->mc_inc_b.upload(inc_b));
  const size_t ab = static_cast<size_t>(s->mc_va) * s->mc_fb * 3 * sizeof(double);
  const size_t ba = static_cast<size_t>(s->mc_vb) * s->mc_fa * 3 * sizeof(double);
  PD_CUDA(s->mc_force_ab.allocate(ab));
  PD_CUDA(s->mc_bary_ab.allocate(ab));
  PD_CUDA(s->mc_force_ba.allocate(ba));
  PD_CUDA(s->mc_bary_ba.allocate(ba));
  PD_CUDA(s->mc_force.allocate(static_cast<size_t>(3) * s->n * sizeof(double)));
  PD_CUDA(s->mc_pairs.allocate(sizeof(int)));
  s->has_mesh_contact = true;
  return PD_OK;
}

extern "C" int pd_mesh_contact_force(PdSolver* s, const double* q, const double* v, double* force, int32_t* pairs,
                                     void* stream) {
  if (s == nullptr || q == nullptr || v == nullptr) return pd_set_error(PD_ERR_INVALID, "null argument");
  if (!s->has_mesh_contact) return pd_set_error(PD_ERR_STATE, "the solver has no mesh_contact");
  PD_CUDA(cudaSetDevice(s->device));
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (int status = pd_evaluate_mesh_contact(s, q, v, 1, st)) return status;
  if (force != nullptr) {
    PD_CUDA(cudaMemcpyAsync(force, s->mc_force.ptr, s->mc_force.bytes, cudaMemcpyDeviceToDevice, st));
  }
  if (pairs != nullptr) {
    PD_CUDA(cudaMemcpyAsync(pairs, s->mc_pairs.ptr, sizeof(int), cudaMemcpyDeviceToHost, st));
    PD_CUDA(cudaStreamSynchronize(st));
  }
  return PD_OK;
}

extern "C" int pd_mesh_contact_pairs(PdSolver* s, int32_t* pairs, void* stream) {
  if (s == nullptr || pairs == nullptr) return pd_set_error(PD_ERR_INVALID, "null argument");
  if (!s->has_mesh_contact) return pd_set_error(PD_ERR_STATE, "the solver has no mesh_contact");
  PD_CUDA(cudaSetDevice(s->device));
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  PD_CUDA(cudaMemcpyAsync(pairs, s->mc_pairs.ptr, sizeof(int), cudaMemcpyDeviceToHost, st));
  PD_CUDA(cudaStreamSynchronize(st));
  return PD_OK;
}
