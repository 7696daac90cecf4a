// Synthetic pressure-correction systems for tests and benchmarks.
//
// Finite-volume two-point-flux matrices on a jittered box mesh of the unit cube:
// hexahedra, or each hexahedron split into six tetrahedra around its main
// diagonal (the same six-tet split as the reference's make_box_tet,
// src/kutta/io/generators.cpp:10-96). Cells are renumbered by reverse
// Cuthill-McKee (the reference renumbers with the same algorithm before it
// assembles the pressure matrix, src/kutta/mesh/topology.cpp:148-230), then the
// symmetric M-matrix is assembled the way the reference's pressure assembly
// stores it: float off-diagonals -a_f and an upward-rounded float diagonal, so
// every stored row sum is >= 0 (src/kutta/fv/steady_solver.cpp:552-575).
//
// Also the reference's own linear-algebra test matrices (poisson(),
// tests/linalg/matrices.hpp:17-62) and a non-symmetric upwind
// convection-diffusion twin on the same mesh.
//
// All randomness comes from a seeded splitmix64 stream; a seed fully fixes a
// system.
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef struct {
  int n, nnz;
  int* row_ptr;   // n + 1
  int* col;       // nnz, sorted per row
  int* diag;      // n
  double* val;    // nnz, every value exactly representable as float
  float* b;       // n, right-hand side
  double* volume; // n, cell volumes
  int* new_to_old;  // n, the renumbering applied (identity when none)
  int faces;        // interior faces
  double* centroid; // 3n, cell centroids (x, y, z) in the stored order; NULL for poisson
  double* boundary; // n, the Dirichlet boundary term in each diagonal; NULL for poisson
  double* geometry; // nnz, the face's geometric coefficient |A_f| / |c_N - c_P| per
                    // off-diagonal entry (0 on the diagonal); NULL for poisson
} kh_system;

// ---------------------------------------------------------------- random ----
static uint64_t splitmix(uint64_t* s) {
  uint64_t z = (*s += 0x9e3779b97f4a7c15ULL);
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
  return z ^ (z >> 31);
}
static double uniform01(uint64_t* s) { return (double)(splitmix(s) >> 11) * 0x1.0p-53; }
static double normal01(uint64_t* s) {
  double u1 = uniform01(s), u2 = uniform01(s);
  if (u1 < 1e-300) u1 = 1e-300;
  return sqrt(-2.0 * log(u1)) * cos(6.283185307179586 * u2);
}

// Upward-rounded float of a long-double sum: the smallest float >= value.
static float float_up(long double value) {
  float f = (float)value;
  if ((long double)f < value) f = nextafterf(f, INFINITY);
  return f;
}

void kh_free(kh_system* s) {
  if (!s) return;
  free(s->row_ptr); free(s->col); free(s->diag); free(s->val);
  free(s->b); free(s->volume); free(s->new_to_old); free(s->centroid); free(s->boundary);
  free(s->geometry);
  free(s);
}

// ------------------------------------------------------- reference poisson ----
// Restates tests/linalg/matrices.hpp:13-62 (hash, poisson) from the reference.
static uint32_t ref_hash(uint32_t x) {
  x ^= x >> 16; x *= 0x7feb352dU; x ^= x >> 15; x *= 0x846ca68bU; return x ^ (x >> 16);
}
uint32_t kh_hash(uint32_t x) { return ref_hash(x); }

kh_system* kh_poisson(int nx, int ny, int nz, double anisotropy, int random, int neumann,
                      double wind) {
  kh_system* s = (kh_system*)calloc(1, sizeof(kh_system));
  const int n = nx * ny * nz;
  const int dims[3] = {nx, ny, nz};
  const int strides[3] = {1, nx, nx * ny};
  const int dimension = nz == 1 ? 2 : 3;
  s->n = n;
  s->row_ptr = (int*)malloc(sizeof(int) * (size_t)(n + 1));
  s->diag = (int*)malloc(sizeof(int) * (size_t)(n > 0 ? n : 1));
  const size_t cap = (size_t)n * (2 * dimension + 1) + 1;
  s->col = (int*)malloc(sizeof(int) * cap);
  s->val = (double*)malloc(sizeof(double) * cap);
  s->b = (float*)calloc((size_t)(n > 0 ? n : 1), sizeof(float));
  s->volume = (double*)malloc(sizeof(double) * (size_t)(n > 0 ? n : 1));
  s->new_to_old = (int*)malloc(sizeof(int) * (size_t)(n > 0 ? n : 1));
  int nnz = 0;
  s->row_ptr[0] = 0;
  for (int i = 0; i < n; ++i) {
    int cols[8];
    double vals[8];
    int count = 0;
    double diagonal = 0;
    for (int d = 0; d < dimension; ++d) {
      const int coord = (i / strides[d]) % dims[d];
      for (int sign = -1; sign <= 1; sign += 2) {
        const int j = i + sign * strides[d];
        const int inside = coord + sign >= 0 && coord + sign < dims[d];
        double weight = d == 0 ? anisotropy : 1;
        if (random && inside) {
          const uint32_t lo = (uint32_t)(i < j ? i : j), hi = (uint32_t)(i < j ? j : i);
          const uint32_t key = ref_hash(lo ^ (ref_hash(hi) + 0x9e3779b9U));
          weight *= 0.1 + 9.9 * (double)(key % 1000) / 999;
        }
        if (inside) { cols[count] = j; vals[count] = -weight; ++count; }
        if (inside || !neumann) diagonal += weight;
      }
    }
    if (wind != 0) {
      diagonal += wind;
      if (i % nx != 0)
        for (int k = 0; k < count; ++k)
          if (cols[k] == i - 1) vals[k] -= wind;
    }
    cols[count] = i; vals[count] = diagonal; ++count;
    // insertion sort by column
    for (int a = 1; a < count; ++a)
      for (int b2 = a; b2 > 0 && cols[b2 - 1] > cols[b2]; --b2) {
        int tc = cols[b2]; cols[b2] = cols[b2 - 1]; cols[b2 - 1] = tc;
        double tv = vals[b2]; vals[b2] = vals[b2 - 1]; vals[b2 - 1] = tv;
      }
    for (int k = 0; k < count; ++k) {
      if (cols[k] == i) s->diag[i] = nnz;
      s->col[nnz] = cols[k];
      s->val[nnz] = (double)(float)vals[k];
      ++nnz;
    }
    s->row_ptr[i + 1] = nnz;
    s->volume[i] = 1.0;
    s->new_to_old[i] = i;
  }
  s->nnz = nnz;
  return s;
}

// ------------------------------------------------------------------ mesh ----
typedef struct { double x, y, z; } v3;
static v3 sub(v3 a, v3 b) { v3 r = {a.x - b.x, a.y - b.y, a.z - b.z}; return r; }
static v3 add(v3 a, v3 b) { v3 r = {a.x + b.x, a.y + b.y, a.z + b.z}; return r; }
static v3 scale(v3 a, double s) { v3 r = {a.x * s, a.y * s, a.z * s}; return r; }
static v3 cross(v3 a, v3 b) {
  v3 r = {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
  return r;
}
static double dot3(v3 a, v3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static double norm3(v3 a) { return sqrt(dot3(a, a)); }

// Grid coordinates along one axis: uniform, or (z only) a band of `layers`
// geometric layers at 0 with first height h/aspect and growth `ratio`, the
// rest uniform.
static void axis(double* c, int cells, int band_layers, double aspect, double ratio) {
  if (band_layers <= 0 || band_layers >= cells) {
    for (int i = 0; i <= cells; ++i) c[i] = (double)i / cells;
    return;
  }
  const double h = 1.0 / cells;
  double dz = h / aspect, z = 0;
  c[0] = 0;
  for (int k = 1; k <= band_layers; ++k) { z += dz; c[k] = z; dz *= ratio; }
  const int rest = cells - band_layers;
  for (int k = 1; k <= rest; ++k) c[band_layers + k] = z + (1.0 - z) * k / rest;
}

// LSD radix sort of (key, value) pairs by a 64-bit key.
static void radix_sort(uint64_t* key, int64_t* value, size_t n) {
  uint64_t* k2 = (uint64_t*)malloc(sizeof(uint64_t) * n);
  int64_t* v2 = (int64_t*)malloc(sizeof(int64_t) * n);
  for (int shift = 0; shift < 64; shift += 16) {
    size_t count[65537];
    memset(count, 0, sizeof(count));
    int any = 0;
    for (size_t i = 0; i < n; ++i) {
      const unsigned d = (unsigned)((key[i] >> shift) & 0xffff);
      ++count[d + 1];
      any |= d != 0;
    }
    if (!any) continue;
    for (int d = 0; d < 65536; ++d) count[d + 1] += count[d];
    for (size_t i = 0; i < n; ++i) {
      const unsigned d = (unsigned)((key[i] >> shift) & 0xffff);
      const size_t at = count[d]++;
      k2[at] = key[i];
      v2[at] = value[i];
    }
    memcpy(key, k2, sizeof(uint64_t) * n);
    memcpy(value, v2, sizeof(int64_t) * n);
  }
  free(k2); free(v2);
}

typedef struct {
  int cells, faces_int, faces_bnd;
  v3* centroid;     // cells
  double* volume;   // cells
  int *owner, *neighbour;  // interior faces
  v3 *area, *fcentre;      // interior faces (area points owner -> neighbour)
  int* b_owner;            // boundary faces
  v3 *b_area, *b_centre;   // boundary faces (outward)
} kh_mesh;

static void mesh_free(kh_mesh* m) {
  free(m->centroid); free(m->volume); free(m->owner); free(m->neighbour);
  free(m->area); free(m->fcentre); free(m->b_owner); free(m->b_area); free(m->b_centre);
}

// Six tetrahedra per hexahedron around the 0-6 diagonal (vertex order
// 0:(0,0,0) 1:(1,0,0) 2:(1,1,0) 3:(0,1,0) 4:(0,0,1) 5:(1,0,1) 6:(1,1,1) 7:(0,1,1)).
static const int kTets[6][4] = {{0, 1, 2, 6}, {0, 2, 3, 6}, {0, 3, 7, 6},
                                {0, 7, 4, 6}, {0, 4, 5, 6}, {0, 5, 1, 6}};

static int build_mesh(kh_mesh* m, int nx, int ny, int nz, int tet, double jitter,
                      int band_layers, double aspect, double ratio, uint64_t* rng) {
  const int px = nx + 1, py = ny + 1, pz = nz + 1;
  const size_t np = (size_t)px * py * pz;
  v3* p = (v3*)malloc(sizeof(v3) * np);
  double* cx = (double*)malloc(sizeof(double) * px);
  double* cy = (double*)malloc(sizeof(double) * py);
  double* cz = (double*)malloc(sizeof(double) * pz);
  axis(cx, nx, 0, 1, 1);
  axis(cy, ny, 0, 1, 1);
  axis(cz, nz, band_layers, aspect, ratio);
  for (int k = 0; k < pz; ++k)
    for (int j = 0; j < py; ++j)
      for (int i = 0; i < px; ++i) {
        v3 q = {cx[i], cy[j], cz[k]};
        const int interior = i > 0 && i < nx && j > 0 && j < ny && k > 0 && k < nz;
        const double ux = uniform01(rng), uy = uniform01(rng), uz = uniform01(rng);
        if (interior && jitter > 0) {
          // +-jitter of the smaller adjacent spacing along each axis.
          const double hx = fmin(cx[i] - cx[i - 1], cx[i + 1] - cx[i]);
          const double hy = fmin(cy[j] - cy[j - 1], cy[j + 1] - cy[j]);
          const double hz = fmin(cz[k] - cz[k - 1], cz[k + 1] - cz[k]);
          q.x += jitter * hx * (2 * ux - 1);
          q.y += jitter * hy * (2 * uy - 1);
          q.z += jitter * hz * (2 * uz - 1);
        }
        p[((size_t)k * py + j) * px + i] = q;
      }
  free(cx); free(cy); free(cz);
  if ((double)np * (double)np * (double)np >= 1.8e19) { free(p); return -1; }
  const size_t hexes = (size_t)nx * ny * nz;
  const int per = tet ? 6 : 1;
  const size_t cells = hexes * per;
  if (cells > 0x7fffffffULL / 8) { free(p); return -1; }
  m->cells = (int)cells;
  m->centroid = (v3*)malloc(sizeof(v3) * cells);
  m->volume = (double*)malloc(sizeof(double) * cells);
  // Face keys: each cell face, key = its sorted vertex ids in radix np (three for
  // triangles; a quad's two smallest ids and its largest identify it). np^3 must
  // fit in 64 bits, which holds up to 2.6M points.
  const int fpc = tet ? 4 : 6;
  const size_t nf = cells * fpc;
  uint64_t* key = (uint64_t*)malloc(sizeof(uint64_t) * nf);
  int64_t* who = (int64_t*)malloc(sizeof(int64_t) * nf);
  int* fverts = (int*)malloc(sizeof(int) * nf * 4);  // face vertex ids, oriented outward
  static const int kHexFaces[6][4] = {{0, 3, 2, 1}, {4, 5, 6, 7}, {0, 1, 5, 4},
                                      {2, 3, 7, 6}, {0, 4, 7, 3}, {1, 2, 6, 5}};
  for (int k = 0; k < nz; ++k)
    for (int j = 0; j < ny; ++j)
      for (int i = 0; i < nx; ++i) {
        const size_t h = ((size_t)k * ny + j) * nx + i;
        int v[8];
        const int di[8] = {0, 1, 1, 0, 0, 1, 1, 0}, dj[8] = {0, 0, 1, 1, 0, 0, 1, 1},
                  dk[8] = {0, 0, 0, 0, 1, 1, 1, 1};
        for (int a = 0; a < 8; ++a) v[a] = (int)(((size_t)(k + dk[a]) * py + (j + dj[a])) * px + (i + di[a]));
        for (int t = 0; t < per; ++t) {
          const size_t c = h * per + t;
          if (tet) {
            const int a0 = v[kTets[t][0]], a1 = v[kTets[t][1]], a2 = v[kTets[t][2]], a3 = v[kTets[t][3]];
            const v3 P0 = p[a0], P1 = p[a1], P2 = p[a2], P3 = p[a3];
            double vol = dot3(sub(P1, P0), cross(sub(P2, P0), sub(P3, P0))) / 6.0;
            int tv[4] = {a0, a1, a2, a3};
            if (vol < 0) { int t2 = tv[1]; tv[1] = tv[2]; tv[2] = t2; vol = -vol; }
            m->volume[c] = vol;
            m->centroid[c] = scale(add(add(P0, P1), add(P2, P3)), 0.25);
            // Faces opposite each vertex, oriented outward for positive orientation.
            static const int kOpp[4][3] = {{1, 3, 2}, {0, 2, 3}, {0, 3, 1}, {0, 1, 2}};
            for (int f = 0; f < 4; ++f) {
              int a = tv[kOpp[f][0]], b = tv[kOpp[f][1]], d = tv[kOpp[f][2]];
              const size_t e = c * 4 + f;
              fverts[e * 4 + 0] = a; fverts[e * 4 + 1] = b; fverts[e * 4 + 2] = d; fverts[e * 4 + 3] = -1;
              int s0 = a, s1 = b, s2 = d, tmp;
              if (s0 > s1) { tmp = s0; s0 = s1; s1 = tmp; }
              if (s1 > s2) { tmp = s1; s1 = s2; s2 = tmp; }
              if (s0 > s1) { tmp = s0; s0 = s1; s1 = tmp; }
              key[e] = ((uint64_t)s0 * np + (uint64_t)s1) * np + (uint64_t)s2;
              who[e] = (int64_t)e;
            }
          } else {
            double vol = 0;
            for (int t2 = 0; t2 < 6; ++t2) {
              const v3 P0 = p[v[kTets[t2][0]]], P1 = p[v[kTets[t2][1]]], P2 = p[v[kTets[t2][2]]], P3 = p[v[kTets[t2][3]]];
              vol += fabs(dot3(sub(P1, P0), cross(sub(P2, P0), sub(P3, P0)))) / 6.0;
            }
            m->volume[c] = vol;
            v3 cen = {0, 0, 0};
            for (int a = 0; a < 8; ++a) cen = add(cen, p[v[a]]);
            m->centroid[c] = scale(cen, 0.125);
            for (int f = 0; f < 6; ++f) {
              const size_t e = c * 6 + f;
              int q[4];
              for (int a = 0; a < 4; ++a) { q[a] = v[kHexFaces[f][a]]; fverts[e * 4 + a] = q[a]; }
              // sort 4 ids
              for (int a = 1; a < 4; ++a)
                for (int b2 = a; b2 > 0 && q[b2 - 1] > q[b2]; --b2) { int t3 = q[b2]; q[b2] = q[b2 - 1]; q[b2 - 1] = t3; }
              key[e] = ((uint64_t)q[0] * np + (uint64_t)q[1]) * np + (uint64_t)q[3];
              who[e] = (int64_t)e;
            }
          }
        }
      }
  radix_sort(key, who, nf);
  size_t ni = 0, nb = 0;
  for (size_t a = 0; a < nf;) {
    if (a + 1 < nf && key[a + 1] == key[a]) { ++ni; a += 2; }
    else { ++nb; a += 1; }
  }
  m->faces_int = (int)ni;
  m->faces_bnd = (int)nb;
  m->owner = (int*)malloc(sizeof(int) * (ni ? ni : 1));
  m->neighbour = (int*)malloc(sizeof(int) * (ni ? ni : 1));
  m->area = (v3*)malloc(sizeof(v3) * (ni ? ni : 1));
  m->fcentre = (v3*)malloc(sizeof(v3) * (ni ? ni : 1));
  m->b_owner = (int*)malloc(sizeof(int) * (nb ? nb : 1));
  m->b_area = (v3*)malloc(sizeof(v3) * (nb ? nb : 1));
  m->b_centre = (v3*)malloc(sizeof(v3) * (nb ? nb : 1));
  size_t fi = 0, fb = 0;
  for (size_t a = 0; a < nf;) {
    const size_t e = (size_t)who[a];
    const int c = (int)(e / fpc);
    const int* fv = fverts + e * 4;
    v3 area, centre;
    if (tet) {
      area = scale(cross(sub(p[fv[1]], p[fv[0]]), sub(p[fv[2]], p[fv[0]])), 0.5);
      centre = scale(add(add(p[fv[0]], p[fv[1]]), p[fv[2]]), 1.0 / 3.0);
    } else {
      area = scale(cross(sub(p[fv[2]], p[fv[0]]), sub(p[fv[3]], p[fv[1]])), 0.5);
      centre = scale(add(add(p[fv[0]], p[fv[1]]), add(p[fv[2]], p[fv[3]])), 0.25);
    }
    // Orient outward from cell c: the area must point away from its centroid.
    if (dot3(area, sub(centre, m->centroid[c])) < 0) area = scale(area, -1);
    if (a + 1 < nf && key[a + 1] == key[a]) {
      const int c2 = (int)((size_t)who[a + 1] / fpc);
      const int lo = c < c2 ? c : c2, hi = c < c2 ? c2 : c;
      m->owner[fi] = lo;
      m->neighbour[fi] = hi;
      m->area[fi] = lo == c ? area : scale(area, -1);
      m->fcentre[fi] = centre;
      ++fi;
      a += 2;
    } else {
      m->b_owner[fb] = c;
      m->b_area[fb] = area;
      m->b_centre[fb] = centre;
      ++fb;
      a += 1;
    }
  }
  free(key); free(who); free(fverts); free(p);
  return 0;
}

// Reverse Cuthill-McKee over the cell adjacency: seeds in increasing degree
// (stable), breadth-first with unvisited neighbours in increasing degree
// (stable), each component reversed. Returns new_to_old.
static int* rcm(int n, const int* off, const int* adj) {
  int* order = (int*)malloc(sizeof(int) * (size_t)n);
  int* seeds = (int*)malloc(sizeof(int) * (size_t)n);
  char* seen = (char*)calloc((size_t)n, 1);
  int* queue = (int*)malloc(sizeof(int) * (size_t)n);
  int maxdeg = 0;
  for (int c = 0; c < n; ++c) if (off[c + 1] - off[c] > maxdeg) maxdeg = off[c + 1] - off[c];
  // counting sort of seeds by degree (stable)
  int* cnt = (int*)calloc((size_t)maxdeg + 2, sizeof(int));
  for (int c = 0; c < n; ++c) ++cnt[off[c + 1] - off[c] + 1];
  for (int d = 0; d <= maxdeg; ++d) cnt[d + 1] += cnt[d];
  for (int c = 0; c < n; ++c) seeds[cnt[off[c + 1] - off[c]]++] = c;
  free(cnt);
  int* row = (int*)malloc(sizeof(int) * ((size_t)maxdeg + 1));
  int filled = 0;
  for (int si = 0; si < n; ++si) {
    const int seed = seeds[si];
    if (seen[seed]) continue;
    int head = 0, tail = 0;
    queue[tail++] = seed;
    seen[seed] = 1;
    while (head < tail) {
      const int c = queue[head++];
      int m = 0;
      for (int e = off[c]; e < off[c + 1]; ++e)
        if (!seen[adj[e]]) row[m++] = adj[e];
      for (int a = 1; a < m; ++a)  // stable insertion sort by degree
        for (int b2 = a; b2 > 0 && (off[row[b2 - 1] + 1] - off[row[b2 - 1]]) > (off[row[b2] + 1] - off[row[b2]]); --b2) {
          int t = row[b2]; row[b2] = row[b2 - 1]; row[b2 - 1] = t;
        }
      for (int a = 0; a < m; ++a)
        if (!seen[row[a]]) { seen[row[a]] = 1; queue[tail++] = row[a]; }
    }
    for (int a = tail - 1; a >= 0; --a) order[filled++] = queue[a];
  }
  free(row); free(seeds); free(seen); free(queue);
  return order;
}

// Pressure system assembled from face coefficients. kind bits:
//   tet       six tetrahedra per hexahedron
//   renumber  apply RCM (else natural order)
// D per cell = exp(U[ln dmin, ln dmax]); a_f = 0.5 (D_P + D_N) |A_f| / |c_N - c_P|.
// Dirichlet p = 0 on the x = 1 patch: a_b = D_P |A_b| / |c_b - c_P| added to a_P.
// Neumann elsewhere. b_i = N(0,1) V_i.
// convection > 0 instead assembles the non-symmetric twin: first-order upwind
// fluxes of u = curl(sum of 8 seeded Fourier modes of a vector potential),
// normalised to |u|~1, plus diffusion nu = `convection` * |A|/|d|, with the
// diagonal divided by the under-relaxation factor 0.7.
// field_sigma > 0 replaces the per-cell log-uniform D by a smooth log-normal
// field D = exp(field_sigma g(x_c)), g a unit-variance Gaussian random field
// with correlation length field_corr, drawn as 64 random Fourier features:
// g(x) = sqrt(2/64) sum_q cos(w_q . x + p_q), w_q ~ N(0, I / corr^2).
static kh_system* assemble(const kh_mesh* m, int renumber, double dmin, double dmax,
                           double convection, double field_sigma, double field_corr,
                           uint64_t* rng) {
  const int n = m->cells;
  double* D = (double*)malloc(sizeof(double) * (size_t)n);
  if (field_sigma > 0) {
    enum { kFeatures = 64 };
    double w[kFeatures][3], p[kFeatures];
    for (int q = 0; q < kFeatures; ++q) {
      for (int d = 0; d < 3; ++d) w[q][d] = normal01(rng) / field_corr;
      p[q] = 6.283185307179586 * uniform01(rng);
    }
    const double norm = sqrt(2.0 / kFeatures);
    for (int c = 0; c < n; ++c) {
      const v3 x = m->centroid[c];
      double g = 0;
      for (int q = 0; q < kFeatures; ++q) g += cos(w[q][0] * x.x + w[q][1] * x.y + w[q][2] * x.z + p[q]);
      D[c] = exp(field_sigma * norm * g);
    }
  } else {
    const double l0 = log(dmin), l1 = log(dmax);
    for (int c = 0; c < n; ++c) D[c] = exp(l0 + (l1 - l0) * uniform01(rng));
  }
  // Fourier modes of the vector potential for the convective twin.
  double mk[8][3], ma[8][3], mp[8];
  for (int q = 0; q < 8; ++q) {
    for (int d = 0; d < 3; ++d) { mk[q][d] = 6.283185307179586 * (1 + (int)(3 * uniform01(rng))) * (uniform01(rng) < 0.5 ? -1 : 1); ma[q][d] = normal01(rng); }
    mp[q] = 6.283185307179586 * uniform01(rng);
  }
  // adjacency (cells) for RCM
  int* deg = (int*)calloc((size_t)n + 1, sizeof(int));
  for (int f = 0; f < m->faces_int; ++f) { ++deg[m->owner[f] + 1]; ++deg[m->neighbour[f] + 1]; }
  for (int c = 0; c < n; ++c) deg[c + 1] += deg[c];
  int* adj = (int*)malloc(sizeof(int) * (size_t)(2 * m->faces_int + 1));
  int* fill = (int*)malloc(sizeof(int) * (size_t)n);
  memcpy(fill, deg, sizeof(int) * (size_t)n);
  for (int f = 0; f < m->faces_int; ++f) {
    adj[fill[m->owner[f]]++] = m->neighbour[f];
    adj[fill[m->neighbour[f]]++] = m->owner[f];
  }
  free(fill);
  int* new_to_old;
  if (renumber) new_to_old = rcm(n, deg, adj);
  else {
    new_to_old = (int*)malloc(sizeof(int) * (size_t)n);
    for (int c = 0; c < n; ++c) new_to_old[c] = c;
  }
  int* old_to_new = (int*)malloc(sizeof(int) * (size_t)n);
  for (int c = 0; c < n; ++c) old_to_new[new_to_old[c]] = c;
  // Face coefficients (float) for each cell's faces, then CSR rows in new order.
  float* coef_on = (float*)malloc(sizeof(float) * (size_t)(m->faces_int ? m->faces_int : 1));   // off-diag in owner row
  float* coef_no = (float*)malloc(sizeof(float) * (size_t)(m->faces_int ? m->faces_int : 1));   // off-diag in neighbour row
  float* add_o = (float*)malloc(sizeof(float) * (size_t)(m->faces_int ? m->faces_int : 1));     // diagonal share, owner
  float* add_n = (float*)malloc(sizeof(float) * (size_t)(m->faces_int ? m->faces_int : 1));     // diagonal share, neighbour
  double* geo = (double*)malloc(sizeof(double) * (size_t)(m->faces_int ? m->faces_int : 1));   // |A_f| / dist
  for (int f = 0; f < m->faces_int; ++f) {
    const int P = m->owner[f], N = m->neighbour[f];
    const double dist = norm3(sub(m->centroid[N], m->centroid[P]));
    const double A = norm3(m->area[f]);
    geo[f] = A / dist;
    if (convection <= 0) {
      const float a = (float)(0.5 * (D[P] + D[N]) * A / dist);
      coef_on[f] = -a; coef_no[f] = -a; add_o[f] = a; add_n[f] = a;
    } else {
      const v3 x = m->fcentre[f];
      double u[3] = {0, 0, 0};
      for (int q = 0; q < 8; ++q) {
        // u = curl(a * sin(k.x + phase)) = cos(k.x+phase) * (k x a)
        const double ph = mk[q][0] * x.x + mk[q][1] * x.y + mk[q][2] * x.z + mp[q];
        const double cs = cos(ph) / (6.283185307179586 * 3.0);
        u[0] += cs * (mk[q][1] * ma[q][2] - mk[q][2] * ma[q][1]);
        u[1] += cs * (mk[q][2] * ma[q][0] - mk[q][0] * ma[q][2]);
        u[2] += cs * (mk[q][0] * ma[q][1] - mk[q][1] * ma[q][0]);
      }
      const double F = u[0] * m->area[f].x + u[1] * m->area[f].y + u[2] * m->area[f].z;
      const double dif = convection * A / dist;
      coef_on[f] = (float)(-(dif + fmax(-F, 0.0)));
      coef_no[f] = (float)(-(dif + fmax(F, 0.0)));
      add_o[f] = (float)(dif + fmax(F, 0.0));
      add_n[f] = (float)(dif + fmax(-F, 0.0));
    }
  }
  // Boundary contributions per cell (Dirichlet on x = 1; outflow for the twin).
  long double* bnd = (long double*)calloc((size_t)n, sizeof(long double));
  for (int f = 0; f < m->faces_bnd; ++f) {
    const int P = m->b_owner[f];
    const v3 A = m->b_area[f];
    const double An = norm3(A);
    const int dirichlet = m->b_centre[f].x > 1.0 - 1e-12 && A.x > 0.9 * An;
    if (convection <= 0) {
      if (dirichlet) bnd[P] += (float)(D[P] * An / norm3(sub(m->b_centre[f], m->centroid[P])));
    } else {
      if (dirichlet) bnd[P] += (float)(convection * An / norm3(sub(m->b_centre[f], m->centroid[P])));
    }
  }
  kh_system* s = (kh_system*)calloc(1, sizeof(kh_system));
  s->n = n;
  s->faces = m->faces_int;
  s->nnz = n + 2 * m->faces_int;
  s->row_ptr = (int*)malloc(sizeof(int) * (size_t)(n + 1));
  s->col = (int*)malloc(sizeof(int) * (size_t)s->nnz);
  s->val = (double*)malloc(sizeof(double) * (size_t)s->nnz);
  s->diag = (int*)malloc(sizeof(int) * (size_t)n);
  s->b = (float*)malloc(sizeof(float) * (size_t)n);
  s->volume = (double*)malloc(sizeof(double) * (size_t)n);
  s->centroid = (double*)malloc(sizeof(double) * 3 * (size_t)n);
  s->boundary = (double*)malloc(sizeof(double) * (size_t)n);
  s->geometry = (double*)malloc(sizeof(double) * (size_t)s->nnz);
  s->new_to_old = new_to_old;
  // faces per old cell
  int* foff = deg;  // reuse adjacency offsets: same counts per cell
  int* fface = (int*)malloc(sizeof(int) * (size_t)(2 * m->faces_int + 1));
  int* cur = (int*)malloc(sizeof(int) * (size_t)n);
  memcpy(cur, foff, sizeof(int) * (size_t)n);
  for (int f = 0; f < m->faces_int; ++f) {
    fface[cur[m->owner[f]]++] = f;
    fface[cur[m->neighbour[f]]++] = f;
  }
  free(cur);
  int nnz = 0;
  s->row_ptr[0] = 0;
  typedef struct { int col; float v; double g; } ent;
  ent* row = (ent*)malloc(sizeof(ent) * 64);
  for (int r = 0; r < n; ++r) {
    const int c = new_to_old[r];
    int cnt = 0;
    long double dsum = bnd[c];
    for (int e = foff[c]; e < foff[c + 1]; ++e) {
      const int f = fface[e];
      const int own = m->owner[f] == c;
      const int other = own ? m->neighbour[f] : m->owner[f];
      row[cnt].col = old_to_new[other];
      row[cnt].v = own ? coef_on[f] : coef_no[f];
      row[cnt].g = geo[f];
      dsum += own ? add_o[f] : add_n[f];
      ++cnt;
    }
    float dval;
    if (convection <= 0) {
      // Row sum of stored floats >= 0: diagonal is the upward-rounded float of the
      // exact off-diagonal magnitudes plus the boundary term.
      long double off = bnd[c];
      for (int a = 0; a < cnt; ++a) off += -(long double)row[a].v;
      dval = float_up(off);
    } else {
      dval = (float)(dsum / 0.7L);
    }
    row[cnt].col = r; row[cnt].v = dval; row[cnt].g = 0.0; ++cnt;
    for (int a = 1; a < cnt; ++a)
      for (int b2 = a; b2 > 0 && row[b2 - 1].col > row[b2].col; --b2) { ent t = row[b2]; row[b2] = row[b2 - 1]; row[b2 - 1] = t; }
    for (int a = 0; a < cnt; ++a) {
      if (row[a].col == r) s->diag[r] = nnz;
      s->col[nnz] = row[a].col;
      s->val[nnz] = (double)row[a].v;
      s->geometry[nnz] = row[a].g;
      ++nnz;
    }
    s->row_ptr[r + 1] = nnz;
    s->volume[r] = m->volume[c];
    s->centroid[3 * (size_t)r] = m->centroid[c].x;
    s->centroid[3 * (size_t)r + 1] = m->centroid[c].y;
    s->centroid[3 * (size_t)r + 2] = m->centroid[c].z;
    s->boundary[r] = (double)bnd[c];
    s->b[r] = (float)(normal01(rng) * m->volume[c]);
  }
  free(row); free(fface); free(bnd); free(coef_on); free(coef_no); free(add_o); free(add_n);
  free(geo);
  free(adj); free(deg); free(old_to_new); free(D);
  return s;
}

// Build a pressure (convection <= 0) or convection-diffusion (convection = nu > 0)
// system on a jittered nx*ny*nz box, hexahedra (tet = 0) or six tets per hex.
// band_layers > 0 grades the first layers at z = 0 (first height h/aspect, growth
// ratio). Returns NULL on invalid sizes.
// coeff_seed != 0 draws the coefficients (and right-hand side) from a stream of
// its own, so one mesh can carry several coefficient fields; 0 continues the
// mesh's stream.
kh_system* kh_box_system(int nx, int ny, int nz, int tet, double jitter, int band_layers,
                         double aspect, double ratio, double dmin, double dmax,
                         double convection, int renumber, uint64_t seed, uint64_t coeff_seed,
                         double field_sigma, double field_corr) {
  if (nx < 1 || ny < 1 || nz < 1) return NULL;
  uint64_t rng = seed * 0x2545F4914F6CDD1DULL + 0x1234567ULL;
  kh_mesh m;
  memset(&m, 0, sizeof(m));
  if (build_mesh(&m, nx, ny, nz, tet, jitter, band_layers, aspect, ratio, &rng) != 0) return NULL;
  if (coeff_seed != 0) rng = coeff_seed * 0x9E3779B97F4A7C15ULL + 0x7654321ULL;
  kh_system* s = assemble(&m, renumber, dmin, dmax, convection, field_sigma, field_corr, &rng);
  mesh_free(&m);
  return s;
}
