/*
 * gg_oracle_gen.c -- TEST INFRASTRUCTURE ONLY (inputs for the checker and the
 * reference's own build, never the product).
 *
 * Builds the synthetic inputs on the host without the GPU library, so that a
 * process timing the reference (bench.py --impl reference) maps no library of
 * the product:
 *   - or_gen_rmat: the seeded R-MAT generator the library ships
 *     (gg_gen_rmat), restated: SplitMix64 keyed by (seed, edge index), one
 *     quadrant choice per level from 32-bit draws against the a, a+b, a+b+c
 *     thresholds scaled by 2^32; self-loops dropped, rows sorted and
 *     de-duplicated.  The tests check it against gg_gen_rmat edge for edge.
 *   - or_add_weights: the (seed, src, dst) hash weights of
 *     gg_host_graph_add_weights.
 *   - or_write_gr: Galois .gr v1, the layout graphgrind/IO.h:365-450 reads
 *     (header {1, edge bytes, n, m}, u64 row ends, u32 destinations padded to
 *     an even count, u32 weights).
 *   - or_csc: the in-edge CSC of a CSR (in-lists ascending by source), the
 *     transpose every oracle graph carries.
 * Rows are built in parallel (OpenMP); the results do not depend on the
 * thread count.
 */
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "gg_oracle.h"

static uint64_t sm64(uint64_t z) {
  z += 0x9e3779b97f4a7c15ULL;
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
  return z ^ (z >> 31);
}

typedef struct {
  int scale;
  uint64_t ta, tab, tabc, base;
} rmat_t;

static void rmat_edge(const rmat_t* r, uint64_t i, uint32_t* u, uint32_t* v) {
  const uint64_t key = sm64(r->base + i);
  uint32_t s = 0, d = 0;
  uint64_t w = 0;
  for (int l = 0; l < r->scale; l++) {
    if ((l & 1) == 0) w = sm64(key + (uint64_t)l);
    const uint64_t x = (l & 1) ? (w >> 32) : (w & 0xffffffffULL);
    const uint32_t q = x < r->ta ? 0u : x < r->tab ? 1u : x < r->tabc ? 2u : 3u;
    s = (s << 1) | (q >> 1);
    d = (d << 1) | (q & 1u);
  }
  *u = s;
  *v = d;
}

static int cmp_u32(const void* a, const void* b) {
  const uint32_t x = *(const uint32_t*)a, y = *(const uint32_t*)b;
  return (x > y) - (x < y);
}

static void sort_row(uint32_t* b, uint64_t len) {
  if (len < 32) {
    for (uint64_t i = 1; i < len; i++) {
      uint32_t x = b[i];
      uint64_t j = i;
      while (j > 0 && b[j - 1] > x) {
        b[j] = b[j - 1];
        j--;
      }
      b[j] = x;
    }
  } else {
    qsort(b, len, sizeof(uint32_t), cmp_u32);
  }
}

int or_gen_rmat(int32_t scale, int32_t edge_factor, double a, double b, double c, uint64_t seed,
                int32_t symmetric, uint32_t* offsets, uint32_t** indices, uint64_t* m_out) {
  if (scale < 1 || scale > 31 || edge_factor < 1 || !offsets || !indices || !m_out) return -1;
  rmat_t r;
  const double two32 = 4294967296.0;
  r.scale = scale;
  r.ta = (uint64_t)(a * two32);
  r.tab = (uint64_t)((a + b) * two32);
  r.tabc = (uint64_t)((a + b + c) * two32);
  r.base = sm64(seed ^ 0x52a1d3e7c4b9f601ULL);
  const uint32_t n = 1u << scale;
  const int64_t cnt = (int64_t)((uint64_t)edge_factor << scale);
  uint64_t* off = (uint64_t*)calloc((size_t)n + 1, sizeof(uint64_t));
  if (!off) return -2;
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < cnt; i++) {
    uint32_t u, v;
    rmat_edge(&r, (uint64_t)i, &u, &v);
    if (u == v) continue;
    __atomic_fetch_add(&off[u + 1], 1, __ATOMIC_RELAXED);
    if (symmetric) __atomic_fetch_add(&off[v + 1], 1, __ATOMIC_RELAXED);
  }
  for (uint32_t i = 0; i < n; i++) off[i + 1] += off[i];
  const uint64_t raw = off[n];
  uint32_t* col = (uint32_t*)malloc(sizeof(uint32_t) * (raw ? raw : 1));
  uint64_t* cur = (uint64_t*)malloc(sizeof(uint64_t) * ((size_t)n + 1));
  if (!col || !cur) {
    free(off);
    free(col);
    free(cur);
    return -2;
  }
  memcpy(cur, off, sizeof(uint64_t) * n);
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < cnt; i++) {
    uint32_t u, v;
    rmat_edge(&r, (uint64_t)i, &u, &v);
    if (u == v) continue;
    col[__atomic_fetch_add(&cur[u], 1, __ATOMIC_RELAXED)] = v;
    if (symmetric) col[__atomic_fetch_add(&cur[v], 1, __ATOMIC_RELAXED)] = u;
  }
  /* sort and de-duplicate each row in place; cur[r] = its new length */
#pragma omp parallel for schedule(dynamic, 1024)
  for (int64_t row = 0; row < (int64_t)n; row++) {
    uint32_t* p = col + off[row];
    const uint64_t len = off[row + 1] - off[row];
    sort_row(p, len);
    uint64_t k = 0;
    for (uint64_t j = 0; j < len; j++)
      if (k == 0 || p[j] != p[k - 1]) p[k++] = p[j];
    cur[row] = k;
  }
  uint64_t m = 0;
  for (uint32_t i = 0; i < n; i++) m += cur[i];
  if (m >= (1ULL << 32) - 64) {
    free(off);
    free(col);
    free(cur);
    return -3;
  }
  uint32_t* idx = (uint32_t*)malloc(sizeof(uint32_t) * (m ? m : 1));
  if (!idx) {
    free(off);
    free(col);
    free(cur);
    return -2;
  }
  offsets[0] = 0;
  for (uint32_t i = 0; i < n; i++) offsets[i + 1] = offsets[i] + (uint32_t)cur[i];
#pragma omp parallel for schedule(static)
  for (int64_t row = 0; row < (int64_t)n; row++)
    memcpy(idx + offsets[row], col + off[row], sizeof(uint32_t) * cur[row]);
  free(off);
  free(col);
  free(cur);
  *indices = idx;
  *m_out = m;
  return 0;
}

void or_free(void* p) { free(p); }

int or_add_weights(uint32_t n, const uint32_t* offsets, const uint32_t* indices, int32_t symmetric,
                   int32_t as_float, uint64_t seed, int32_t lo, int32_t hi, void* weights) {
  if (!offsets || !indices || !weights || (!as_float && hi < lo)) return -1;
  const uint64_t base = sm64(seed ^ 0x7f4a7c159e3779b9ULL);
  const uint64_t span = (uint64_t)((int64_t)hi - (int64_t)lo + 1);
#pragma omp parallel for schedule(dynamic, 4096)
  for (int64_t u = 0; u < (int64_t)n; u++) {
    for (uint32_t j = offsets[u]; j < offsets[u + 1]; j++) {
      uint64_t x = (uint64_t)u, y = indices[j];
      if (symmetric && y < x) {
        const uint64_t t = x;
        x = y;
        y = t;
      }
      const uint64_t h = sm64(base + ((x << 32) | y));
      if (as_float)
        ((float*)weights)[j] = (float)((double)((h >> 40) + 1) * (1.0 / 16777216.0));
      else
        ((int32_t*)weights)[j] = (int32_t)(lo + (int64_t)(h % span));
    }
  }
  return 0;
}

int or_csc(uint32_t n, uint64_t m, const uint32_t* out_off, const uint32_t* out_idx, const double* out_w,
           uint32_t* in_off, uint32_t* in_idx, double* in_w) {
  if (!out_off || !out_idx || !in_off || !in_idx) return -1;
  memset(in_off, 0, sizeof(uint32_t) * ((size_t)n + 1));
  for (uint64_t j = 0; j < m; j++) in_off[out_idx[j] + 1]++;
  for (uint32_t i = 0; i < n; i++) in_off[i + 1] += in_off[i];
  uint32_t* cur = (uint32_t*)malloc(sizeof(uint32_t) * ((size_t)n + 1));
  if (!cur) return -2;
  memcpy(cur, in_off, sizeof(uint32_t) * n);
  /* sources in ascending order, so every in-list comes out sorted by source */
  for (uint32_t u = 0; u < n; u++)
    for (uint32_t j = out_off[u]; j < out_off[u + 1]; j++) {
      const uint32_t slot = cur[out_idx[j]]++;
      in_idx[slot] = u;
      if (in_w && out_w) in_w[slot] = out_w[j];
    }
  free(cur);
  return 0;
}

static int put(FILE* f, const void* p, size_t bytes) { return fwrite(p, 1, bytes, f) == bytes ? 0 : -1; }

static int write_one(const char* path, uint32_t n, uint64_t m, const uint32_t* off, const uint32_t* idx,
                     const int32_t* w) {
  FILE* f = fopen(path, "wb");
  if (!f) return -1;
  uint64_t hdr[4] = {1, w ? 4u : 0u, n, m};
  int rc = put(f, hdr, sizeof hdr);
  uint64_t* ends = (uint64_t*)malloc(sizeof(uint64_t) * (n ? n : 1));
  if (!ends) rc = -1;
  for (uint32_t i = 0; !rc && i < n; i++) ends[i] = off[i + 1];
  if (!rc) rc = put(f, ends, sizeof(uint64_t) * n);
  free(ends);
  if (!rc) rc = put(f, idx, sizeof(uint32_t) * m);
  const uint32_t zero = 0;
  if (!rc && (m & 1)) rc = put(f, &zero, 4);
  if (!rc && w) rc = put(f, w, sizeof(int32_t) * m);
  if (fclose(f)) rc = -1;
  return rc;
}

int or_write_gr(const char* path, uint32_t n, uint64_t m, const uint32_t* off, const uint32_t* idx,
                const int32_t* w, int32_t symmetric) {
  int rc = write_one(path, n, m, off, idx, w);
  if (rc || symmetric) return rc;
  /* a directed graph also gets "<path>_t", its transpose, which the
   * reference reads beside the file */
  uint32_t* toff = (uint32_t*)malloc(sizeof(uint32_t) * ((size_t)n + 1));
  uint32_t* tidx = (uint32_t*)malloc(sizeof(uint32_t) * (m ? m : 1));
  int32_t* tw = w ? (int32_t*)malloc(sizeof(int32_t) * (m ? m : 1)) : NULL;
  uint32_t* cur = (uint32_t*)malloc(sizeof(uint32_t) * ((size_t)n + 1));
  char* tp = (char*)malloc(strlen(path) + 3);
  if (!toff || !tidx || (w && !tw) || !cur || !tp) rc = -2;
  if (!rc) {
    memset(toff, 0, sizeof(uint32_t) * ((size_t)n + 1));
    for (uint64_t j = 0; j < m; j++) toff[idx[j] + 1]++;
    for (uint32_t i = 0; i < n; i++) toff[i + 1] += toff[i];
    memcpy(cur, toff, sizeof(uint32_t) * n);
    for (uint32_t u = 0; u < n; u++)
      for (uint32_t j = off[u]; j < off[u + 1]; j++) {
        const uint32_t s = cur[idx[j]]++;
        tidx[s] = u;
        if (tw) tw[s] = w[j];
      }
    strcpy(tp, path);
    strcat(tp, "_t");
    rc = write_one(tp, n, m, toff, tidx, tw);
  }
  free(toff);
  free(tidx);
  free(tw);
  free(cur);
  free(tp);
  return rc;
}
