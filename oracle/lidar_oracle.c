/*
 * lidar_oracle.c -- CPU restatement of the reference Gaussian-LiDAR oracle.
 *
 * TEST INFRASTRUCTURE ONLY: loaded by tests/, __graft_entry__.smoke() and
 * bench.py's cpu_baseline leg (as liboracle_lidar.so); the renderer never
 * uses it.
 *
 * Follows the float64 collect-sort-reduce oracle of the reference,
 * experiments/lidar_cpu_oracle.py:
 *   :28-42   WXYZ quaternion -> rotation (columns are the Gaussian's axes)
 *   :45-88   surfel candidate: normal = axis of the smallest scale, planarity
 *            smallest / min(tangent scales) <= ratio, |cos| >= min_incidence,
 *            plane distance t in [near, far], tangent Mahalanobis q <= sigma^2,
 *            support exp(-q/2), weight = opacity * support * confidence >=
 *            threshold, intensity = clamp(reflectivity * support * |cos|)
 *   :91-190  per (sensor, ray): sensor/scene transforms, candidates sorted by
 *            (t, semantic), up to K returns: first t beyond the previous
 *            cluster end, cluster window max(abs, rel * t), weighted range and
 *            intensity, semantic = largest summed weight (ties -> smallest id)
 * Brute force over every Gaussian of the ray's scene (no acceleration
 * structure, so it is independent of the LBVH it checks).  Sums use
 * Neumaier compensation in place of math.fsum.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#ifdef _OPENMP
#include <omp.h>
#endif

typedef struct lo_config {
  double near_plane;
  double far_plane;
  double support_sigma;
  double detection_threshold;
  double planarity_ratio_max;
  double min_incidence_cos;
  double cluster_abs;
  double cluster_relative;
  double fallback_reflectivity;
} lo_config;

typedef struct lo_scene {
  int64_t scene_id;
  int64_t count;
  const double* means;       /* [G,3] */
  const double* scales;      /* [G,3] */
  const double* rotations;   /* [G,4] WXYZ */
  const double* opacities;   /* [G] */
  const int64_t* semantics;  /* [G] */
  const double* reflectivity; /* [G] or NULL */
  const double* confidence;   /* [G] or NULL */
} lo_scene;

typedef struct candidate {
  double t, w, intensity;
  int64_t semantic;
} candidate;

typedef struct kahan {
  double sum, c;
} kahan;

static void kadd(kahan* k, double v) {
  const double t = k->sum + v;
  if (fabs(k->sum) >= fabs(v)) {
    k->c += (k->sum - t) + v;
  } else {
    k->c += (v - t) + k->sum;
  }
  k->sum = t;
}
static double kget(const kahan* k) { return k->sum + k->c; }

static void rotation_columns(const double* q, double r[3][3]) {
  const double w = q[0], x = q[1], y = q[2], z = q[3];
  /* r[row][col]; column col is the Gaussian's axis col. */
  r[0][0] = 1 - 2 * (y * y + z * z);
  r[0][1] = 2 * (x * y - z * w);
  r[0][2] = 2 * (x * z + y * w);
  r[1][0] = 2 * (x * y + z * w);
  r[1][1] = 1 - 2 * (x * x + z * z);
  r[1][2] = 2 * (y * z - x * w);
  r[2][0] = 2 * (x * z - y * w);
  r[2][1] = 2 * (y * z + x * w);
  r[2][2] = 1 - 2 * (x * x + y * y);
}

static int evaluate(const lo_scene* s, int64_t g, const double* o, const double* d,
                    const lo_config* cfg, candidate* out) {
  const double* sc = s->scales + 3 * g;
  int normal_axis = 0;
  for (int a = 1; a < 3; ++a)
    if (sc[a] < sc[normal_axis]) normal_axis = a;
  int tangent[2], nt = 0;
  for (int a = 0; a < 3; ++a)
    if (a != normal_axis) tangent[nt++] = a;
  const double tmin = fmin(sc[tangent[0]], sc[tangent[1]]);
  if (sc[normal_axis] <= 0 || sc[normal_axis] / tmin > cfg->planarity_ratio_max) return 0;
  double r[3][3];
  rotation_columns(s->rotations + 4 * g, r);
  const double n[3] = {r[0][normal_axis], r[1][normal_axis], r[2][normal_axis]};
  const double denom = n[0] * d[0] + n[1] * d[1] + n[2] * d[2];
  const double incidence = fabs(denom);
  if (incidence < cfg->min_incidence_cos) return 0;
  const double* m = s->means + 3 * g;
  const double t = (n[0] * (m[0] - o[0]) + n[1] * (m[1] - o[1]) + n[2] * (m[2] - o[2])) / denom;
  if (t < cfg->near_plane || t > cfg->far_plane) return 0;
  const double off[3] = {o[0] + t * d[0] - m[0], o[1] + t * d[1] - m[1], o[2] + t * d[2] - m[2]};
  double q = 0.0;
  for (int k = 0; k < 2; ++k) {
    const int a = tangent[k];
    const double c = (off[0] * r[0][a] + off[1] * r[1][a] + off[2] * r[2][a]) / sc[a];
    q += c * c;
  }
  if (q > cfg->support_sigma * cfg->support_sigma) return 0;
  const double support = exp(-0.5 * q);
  const double confidence = s->confidence ? s->confidence[g] : 1.0;
  const double weight = s->opacities[g] * support * confidence;
  if (!isfinite(weight) || weight < cfg->detection_threshold) return 0;
  const double refl = s->reflectivity ? s->reflectivity[g] : cfg->fallback_reflectivity;
  double intensity = refl * support * incidence;
  intensity = fmin(fmax(intensity, 0.0), 1.0);
  out->t = t;
  out->w = weight;
  out->intensity = intensity;
  out->semantic = s->semantics[g];
  return 1;
}

static int cand_cmp(const void* pa, const void* pb) {
  const candidate* a = (const candidate*)pa;
  const candidate* b = (const candidate*)pb;
  if (a->t != b->t) return a->t < b->t ? -1 : 1;
  if (a->semantic != b->semantic) return a->semantic < b->semantic ? -1 : 1;
  return 0;
}

/* Outputs: range/intensity [B,R,K] f64, position [B,R,K,3] f64, semantic
 * [B,R,K] i64, valid [B,R,K] u8, return_count [B,R] i32.  Inactive sensors
 * and rays without a hit keep the caller's initial values (the no-hit
 * contract: +inf, 0, 0, -1, false, 0). Returns 0, -1 on a missing scene,
 * -2 on allocation failure. */
int lo_render(const lo_scene* scenes, int64_t scene_count, const double* dirs, int64_t rays,
              const double* sensor_to_world, const double* scene_to_world,
              const int64_t* scene_ids, int64_t batch, const int64_t* active, int64_t active_count,
              int64_t returns, const lo_config* cfg, int threads, double* range, double* position,
              double* intensity, int64_t* semantic, uint8_t* valid, int32_t* return_count) {
#ifdef _OPENMP
  if (threads > 0) omp_set_num_threads(threads);
#endif
  const int64_t sensors = active ? active_count : batch;
  for (int64_t a = 0; a < sensors; ++a) {
    const int64_t sensor = active ? active[a] : a;
    const lo_scene* scene = NULL;
    for (int64_t k = 0; k < scene_count; ++k)
      if (scenes[k].scene_id == scene_ids[sensor]) scene = &scenes[k];
    if (!scene) return -1;
    const double* st = sensor_to_world + 16 * sensor;
    const double* xt = scene_to_world + 16 * sensor;
    const double wo[3] = {st[3], st[7], st[11]};
    const double rel[3] = {wo[0] - xt[3], wo[1] - xt[7], wo[2] - xt[11]};
    double lo[3];
    for (int i = 0; i < 3; ++i) lo[i] = xt[0 * 4 + i] * rel[0] + xt[1 * 4 + i] * rel[1] + xt[2 * 4 + i] * rel[2];
    int failed = 0;
#pragma omp parallel for schedule(dynamic, 16)
    for (int64_t ray = 0; ray < rays; ++ray) {
      const double* d = dirs + 3 * ray;
      double wd[3], ld[3];
      for (int i = 0; i < 3; ++i) wd[i] = st[i * 4 + 0] * d[0] + st[i * 4 + 1] * d[1] + st[i * 4 + 2] * d[2];
      for (int i = 0; i < 3; ++i) ld[i] = xt[0 * 4 + i] * wd[0] + xt[1 * 4 + i] * wd[1] + xt[2 * 4 + i] * wd[2];
      int64_t cap = 64, n = 0;
      candidate* c = (candidate*)malloc((size_t)cap * sizeof(candidate));
      if (!c) {
        failed = 1;
        continue;
      }
      for (int64_t g = 0; g < scene->count; ++g) {
        candidate cd;
        if (!evaluate(scene, g, lo, ld, cfg, &cd)) continue;
        if (n == cap) {
          cap *= 2;
          candidate* grown = (candidate*)realloc(c, (size_t)cap * sizeof(candidate));
          if (!grown) {
            failed = 1;
            break;
          }
          c = grown;
        }
        c[n++] = cd;
      }
      qsort(c, (size_t)n, sizeof(candidate), cand_cmp);
      double previous_end = cfg->near_plane - 1.0e-12;
      const int64_t base = (sensor * rays + ray) * returns;
      int32_t count = 0;
      int64_t start = 0;
      for (int64_t k = 0; k < returns; ++k) {
        while (start < n && !(c[start].t > previous_end)) ++start;
        if (start >= n) break;
        const double first_t = c[start].t;
        const double end = fmin(cfg->far_plane, first_t + fmax(cfg->cluster_abs, cfg->cluster_relative * first_t));
        kahan tw = {0, 0}, tr = {0, 0}, ti = {0, 0};
        /* label aggregation: the cluster is small; quadratic search is fine */
        int64_t labels[256];
        kahan lw[256];
        int nl = 0;
        int64_t idx = start;
        for (; idx < n && c[idx].t <= end; ++idx) {
          kadd(&tw, c[idx].w);
          kadd(&tr, c[idx].t * c[idx].w);
          kadd(&ti, c[idx].intensity * c[idx].w);
          int slot = -1;
          for (int l = 0; l < nl; ++l)
            if (labels[l] == c[idx].semantic) slot = l;
          if (slot < 0 && nl < 256) {
            slot = nl++;
            labels[slot] = c[idx].semantic;
            lw[slot].sum = 0;
            lw[slot].c = 0;
          }
          if (slot >= 0) kadd(&lw[slot], c[idx].w);
        }
        const double total = kget(&tw);
        const double rng = kget(&tr) / total;
        int best = 0;
        for (int l = 1; l < nl; ++l) {
          const double a = kget(&lw[l]), b = kget(&lw[best]);
          if (a > b || (a == b && labels[l] < labels[best])) best = l;
        }
        range[base + k] = rng;
        intensity[base + k] = kget(&ti) / total;
        semantic[base + k] = labels[best];
        valid[base + k] = 1;
        for (int i = 0; i < 3; ++i) position[(base + k) * 3 + i] = wo[i] + rng * wd[i];
        ++count;
        previous_end = end;
      }
      return_count[sensor * rays + ray] = count;
      free(c);
    }
    if (failed) return -2;
  }
  return 0;
}
