// The wall distance of every cell centre of a 3D mesh on the device: one thread per point,
// the wall faces streamed through shared memory in tiles, each offered to the point's
// candidate list unless a lower bound (the distance to the face's bounding sphere) shows
// it cannot enter; then the exact patch distance over the candidates.  The bound only
// skips faces the ranking would reject, so the candidates are those of the full ranking.
#include "walldist3d.cuh"

namespace jr {

constexpr int WD_THREADS = 128;
constexpr int WD_TILE = 128;

__global__ void k_wall_spheres(const double* __restrict__ quads, int n_faces, double* __restrict__ spheres) {
  const int f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f < n_faces) face_sphere(quads + (size_t)12 * f, spheres + (size_t)4 * f);
}

__global__ void __launch_bounds__(WD_THREADS) k_wall_distance(const double* __restrict__ points, long long n_points,
                                                              const double* __restrict__ quads,
                                                              const double* __restrict__ spheres, int n_faces,
                                                              double* __restrict__ out) {
  __shared__ double tile[WD_TILE * 12];
  __shared__ double sph[WD_TILE * 4];
  const long long i = (long long)blockIdx.x * WD_THREADS + threadIdx.x;
  const bool live = i < n_points;
  const V3 p = live ? v3(points + 3 * i) : V3{0.0, 0.0, 0.0};
  Candidates cand;
  cand.init(n_faces);
  for (int f0 = 0; f0 < n_faces; f0 += WD_TILE) {
    const int m = n_faces - f0 < WD_TILE ? n_faces - f0 : WD_TILE;
    __syncthreads();
    for (int e = threadIdx.x; e < m * 12; e += WD_THREADS) tile[e] = quads[(size_t)12 * f0 + e];
    for (int e = threadIdx.x; e < m * 4; e += WD_THREADS) sph[e] = spheres[(size_t)4 * f0 + e];
    __syncthreads();
    if (!live) continue;
    for (int t = 0; t < m; ++t) offer_face(cand, p, tile + 12 * t, sph + 4 * t, f0 + t);
  }
  if (live) out[i] = n_faces > 0 ? candidates_distance(p, cand, quads) : INFINITY;
}

// points (n, 3) and faces (m, 4, 3) on the device; spheres: m * 4 doubles of scratch
void launch_wall_distance3(const double* points, long long n_points, const double* quads, int n_faces,
                           double* spheres, double* out, cudaStream_t st) {
  if (n_faces > 0) k_wall_spheres<<<(n_faces + 127) / 128, 128, 0, st>>>(quads, n_faces, spheres);
  if (n_points > 0)
    k_wall_distance<<<(unsigned)((n_points + WD_THREADS - 1) / WD_THREADS), WD_THREADS, 0, st>>>(
        points, n_points, quads, spheres, n_faces, out);
}

}  // namespace jr
