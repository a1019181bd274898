// The exact distance from a point to the nearest wall face of a 3D mesh (the wall faces
// as bilinear patches), for the SA model's destruction term: every face ranked by the
// distance to its two triangles (a-b-c and a-c-d; point-triangle distance by barycentric
// projection and the three edges, Ericson, Real-Time Collision Detection, 2005, 5.1.5),
// then the patch distance (Newton on |x(u, v) - p|^2 from the patch centre, kept if it
// lands inside, and the four edges) taken over the CANDIDATES nearest faces -- the
// method of src/jaxrans/mesh/wall3d.py:1-158.  Host-and-device code: the kernel and a
// test-only host harness run the same arithmetic.
#pragma once
#include <cmath>

namespace jr {

constexpr int WD_CANDIDATES = 16;
constexpr int WD_NEWTON = 12;

struct V3 {
  double x, y, z;
};

__host__ __device__ __forceinline__ V3 v3(const double* a) { return {a[0], a[1], a[2]}; }
__host__ __device__ __forceinline__ V3 sub(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__host__ __device__ __forceinline__ double vdot(V3 a, V3 b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }
__host__ __device__ __forceinline__ V3 vcross(V3 a, V3 b) {
  return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}

__host__ __device__ __forceinline__ double segment_distance(V3 p, V3 s, V3 e) {
  const V3 edge = sub(e, s);
  double t = vdot(sub(p, s), edge) / fmax(vdot(edge, edge), 1e-300);
  t = fmin(fmax(t, 0.0), 1.0);
  const V3 r = {p.x - s.x - t * edge.x, p.y - s.y - t * edge.y, p.z - s.z - t * edge.z};
  return sqrt(vdot(r, r));
}

__host__ __device__ __forceinline__ double triangle_distance(V3 p, V3 a, V3 b, V3 c) {
  const V3 ab = sub(b, a), ac = sub(c, a);
  const V3 n = vcross(ab, ac);
  const double nn = vdot(n, n);
  const V3 ap = sub(p, a);
  const double safe = nn > 0.0 ? nn : 1.0;
  const double v = vdot(vcross(ap, ac), n) / safe;
  const double w = vdot(vcross(ab, ap), n) / safe;
  const bool inside = nn > 0.0 && v >= 0.0 && w >= 0.0 && v + w <= 1.0;
  double best = inside ? fabs(vdot(ap, n)) / sqrt(safe) : INFINITY;
  best = fmin(best, segment_distance(p, a, b));
  best = fmin(best, segment_distance(p, b, c));
  best = fmin(best, segment_distance(p, c, a));
  return best;
}

// q: the face's four corners a, b, c, d (12 doubles, round the face)
__host__ __device__ __forceinline__ double face_rank_distance(V3 p, const double* q) {
  const V3 a = v3(q), b = v3(q + 3), c = v3(q + 6), d = v3(q + 9);
  return fmin(triangle_distance(p, a, b, c), triangle_distance(p, a, c, d));
}

__host__ __device__ __forceinline__ double patch_distance(V3 p, const double* q) {
  const V3 a = v3(q), b = v3(q + 3), c = v3(q + 6), d = v3(q + 9);
  const V3 eu = sub(b, a), ev = sub(d, a);
  const V3 w = {a.x - b.x + c.x - d.x, a.y - b.y + c.y - d.y, a.z - b.z + c.z - d.z};
  double u = 0.5, v = 0.5;
  auto point = [&](double uu, double vv) {
    return V3{a.x + uu * eu.x + vv * ev.x + (uu * vv) * w.x - p.x, a.y + uu * eu.y + vv * ev.y + (uu * vv) * w.y - p.y,
              a.z + uu * eu.z + vv * ev.z + (uu * vv) * w.z - p.z};
  };
  for (int it = 0; it < WD_NEWTON; ++it) {
    const V3 xu = {eu.x + v * w.x, eu.y + v * w.y, eu.z + v * w.z};
    const V3 xv = {ev.x + u * w.x, ev.y + u * w.y, ev.z + u * w.z};
    const V3 r = point(u, v);
    const double gu = vdot(r, xu), gv = vdot(r, xv);
    const double huu = vdot(xu, xu), hvv = vdot(xv, xv);
    const double huv = vdot(xu, xv) + vdot(r, w);
    const double det = huu * hvv - huv * huv;
    if (fabs(det) > 1e-300) {
      const double nu = u - (hvv * gu - huv * gv) / det;
      const double nv = v - (huu * gv - huv * gu) / det;
      u = nu;
      v = nv;
    }
    u = fmin(fmax(u, -0.5), 1.5);
    v = fmin(fmax(v, -0.5), 1.5);
  }
  const V3 r = point(u, v);
  const bool inside = u >= 0.0 && u <= 1.0 && v >= 0.0 && v <= 1.0;
  double best = inside ? sqrt(vdot(r, r)) : INFINITY;
  best = fmin(best, segment_distance(p, a, b));
  best = fmin(best, segment_distance(p, b, c));
  best = fmin(best, segment_distance(p, c, d));
  best = fmin(best, segment_distance(p, d, a));
  return best;
}

// The candidate list of one point: the K smallest rank distances seen so far, ascending,
// faces of equal distance in the order they were offered (a stable ranking).
struct Candidates {
  double dist[WD_CANDIDATES];
  int face[WD_CANDIDATES];
  int k;

  __host__ __device__ void init(int n_faces) {
    k = n_faces < WD_CANDIDATES ? n_faces : WD_CANDIDATES;
    for (int j = 0; j < WD_CANDIDATES; ++j) {
      dist[j] = INFINITY;
      face[j] = -1;
    }
  }
  __host__ __device__ double worst() const { return dist[k - 1]; }
  __host__ __device__ void offer(double d, int f) {
    if (!(d < dist[k - 1]) && face[k - 1] >= 0) return;
    int j = k - 1;
    while (j > 0 && (dist[j - 1] > d || face[j - 1] < 0)) {
      dist[j] = dist[j - 1];
      face[j] = face[j - 1];
      --j;
    }
    dist[j] = d;
    face[j] = f;
  }
};

// the sphere (centre, radius) round a face: its corners' mean and the farthest corner
__host__ __device__ __forceinline__ void face_sphere(const double* q, double* out) {
  V3 c = {0.0, 0.0, 0.0};
  for (int k = 0; k < 4; ++k) {
    c.x += 0.25 * q[3 * k];
    c.y += 0.25 * q[3 * k + 1];
    c.z += 0.25 * q[3 * k + 2];
  }
  double r = 0.0;
  for (int k = 0; k < 4; ++k) {
    const V3 e = sub(v3(q + 3 * k), c);
    r = fmax(r, sqrt(vdot(e, e)));
  }
  out[0] = c.x;
  out[1] = c.y;
  out[2] = c.z;
  out[3] = r;
}

// Offer face f (corners q, sphere s) unless the list is full and the distance to the
// sphere, less a rounding margin, already exceeds the worst candidate: such a face's
// rank distance would exceed it too and the offer would be refused.
__host__ __device__ __forceinline__ void offer_face(Candidates& c, V3 p, const double* q, const double* s, int f) {
  if (c.face[c.k - 1] >= 0) {
    const V3 e = sub(p, v3(s));
    const double centre = sqrt(vdot(e, e)), radius = s[3];
    if (centre - radius - 1e-12 * (centre + radius) > c.worst()) return;
  }
  c.offer(face_rank_distance(p, q), f);
}

// the nearest-candidate patch distance once every face has been offered
__host__ __device__ __forceinline__ double candidates_distance(V3 p, const Candidates& c, const double* quads) {
  double best = INFINITY;
  for (int j = 0; j < c.k; ++j)
    if (c.face[j] >= 0) best = fmin(best, patch_distance(p, quads + (size_t)12 * c.face[j]));
  return best;
}

}  // namespace jr
