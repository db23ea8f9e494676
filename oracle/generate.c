/* Test infrastructure, not product code: a CPU restatement of the library's
 * seeded tensor generator (mm-csf_b200/csrc/generate.cu, mmcsf_generate), so
 * that the CPU legs of the benchmark (the reference's MTTKRP_COO_CPU on the
 * host) build their input tensor without loading the CUDA library. Only
 * tests/, __graft_entry__.smoke() and bench.py's CPU-baseline / reference
 * legs use it. The reference itself has no seeded generator (its
 * tools/generate_tensor.py writes .tns text); the benchmark tensors stand in
 * for the FROSTT data of its scripts (scripts/run_all.sh).
 *
 * Definition (the same as the device's): candidate j draws, for every mode m,
 * u = u01(hash3(seed, m + 1, j)); a uniform mode takes floor(u * dim), a
 * Zipf(s) mode takes the first rank whose CDF reaches u, mapped through a
 * seeded Fisher-Yates permutation. The tensor is the first `nnz` candidates,
 * in candidate order, whose coordinates no earlier candidate took; values
 * depend only on the kept candidate's j. Planted-model values are not
 * restated (the benchmark's CPU legs do not use them).
 *
 * Parallel form: candidate keys are computed by T threads; duplicates are
 * resolved by T threads that each own the keys whose hash falls in their
 * share and visit candidates in j order, so the first occurrence of every key
 * wins exactly as in a sequential scan. Rounds draw more candidates until
 * `nnz` are kept. */
#include <math.h>
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef uint64_t u64;
typedef uint32_t u32;

static u64 g_splitmix(u64 x) {
  x += 0x9e3779b97f4a7c15ull;
  x = (x ^ (x >> 30)) * 0xbf58476d1ce4e5b9ull;
  x = (x ^ (x >> 27)) * 0x94d049bb133111ebull;
  return x ^ (x >> 31);
}
static u64 g_hash3(u64 seed, u64 stream, u64 j) { return g_splitmix(g_splitmix(seed ^ (stream * 0xd1b54a32d192ed03ull)) ^ j); }
static double g_u01(u64 h) { return ((double)(h >> 11) + 0.5) * (1.0 / 9007199254740992.0); }

typedef struct {
  int nd;
  u64 seed;
  u64 dims[4];
  int dist[4];
  double* cdf[4];
  u32* perm[4];
  u64 radix[4];
} gen_t;

static u32 g_coord(const gen_t* g, int m, u64 j) {
  const double u = g_u01(g_hash3(g->seed, (u64)m + 1, j));
  const u64 d = g->dims[m];
  if (g->dist[m] == 0) {
    const u64 k = (u64)(u * (double)d);
    return (u32)(k < d ? k : d - 1);
  }
  u64 lo = 0, hi = d - 1;
  const double* c = g->cdf[m];
  while (lo < hi) {
    const u64 mid = (lo + hi) >> 1;
    if (c[mid] < u) lo = mid + 1; else hi = mid;
  }
  return g->perm[m][lo];
}

static u64 g_key(const gen_t* g, u64 j) {
  u64 k = 0;
  for (int m = 0; m < g->nd; ++m) k += (u64)g_coord(g, m, j) * g->radix[m];
  return k;
}

/* ---- round work ---------------------------------------------------------- */
typedef struct {
  const gen_t* g;
  u64 j0, cnt;   /* candidates j0 .. j0+cnt-1 of this round */
  u64* keys;     /* [cnt] */
  unsigned char* kept; /* [cnt] */
  int t, T;
  /* dedup state owned by thread t: open addressing, empty = UINT64_MAX */
  u64** tab;
  u64* cap;
  u64* fill;
  int fail;
} work_t;

static void* g_keys_thread(void* p) {
  work_t* w = (work_t*)p;
  const u64 a = w->cnt * (u64)w->t / (u64)w->T, b = w->cnt * (u64)(w->t + 1) / (u64)w->T;
  for (u64 i = a; i < b; ++i) w->keys[i] = g_key(w->g, w->j0 + i);
  return NULL;
}

static int g_insert(u64** tab, u64* cap, u64* fill, u64 key) {
  if ((*fill + 1) * 10 > *cap * 7) { /* grow to keep the load under 0.7 */
    const u64 ncap = *cap * 2;
    u64* nt = (u64*)malloc(ncap * sizeof(u64));
    if (!nt) return -1;
    memset(nt, 0xff, ncap * sizeof(u64));
    for (u64 i = 0; i < *cap; ++i) {
      const u64 k = (*tab)[i];
      if (k == UINT64_MAX) continue;
      u64 h = g_splitmix(k ^ 0x51ed27u) & (ncap - 1);
      while (nt[h] != UINT64_MAX) h = (h + 1) & (ncap - 1);
      nt[h] = k;
    }
    free(*tab);
    *tab = nt;
    *cap = ncap;
  }
  u64 h = g_splitmix(key ^ 0x51ed27u) & (*cap - 1);
  for (;;) {
    const u64 k = (*tab)[h];
    if (k == key) return 0;
    if (k == UINT64_MAX) {
      (*tab)[h] = key;
      ++*fill;
      return 1;
    }
    h = (h + 1) & (*cap - 1);
  }
}

static void* g_dedup_thread(void* p) {
  work_t* w = (work_t*)p;
  for (u64 i = 0; i < w->cnt; ++i) {
    const u64 k = w->keys[i];
    if ((int)(g_splitmix(k) % (u64)w->T) != w->t) continue;
    const int r = g_insert(&w->tab[w->t], &w->cap[w->t], &w->fill[w->t], k);
    if (r < 0) { w->fail = 1; return NULL; }
    w->kept[i] = (unsigned char)r;
  }
  return NULL;
}

typedef struct {
  const gen_t* g;
  const u64* cand;
  u64 n;
  int val_dist;
  u32** inds;
  float* vals;
  int t, T;
} emit_t;

static void* g_emit_thread(void* p) {
  emit_t* e = (emit_t*)p;
  const u64 a = e->n * (u64)e->t / (u64)e->T, b = e->n * (u64)(e->t + 1) / (u64)e->T;
  for (u64 x = a; x < b; ++x) {
    const u64 j = e->cand[x];
    for (int m = 0; m < e->g->nd; ++m) e->inds[m][x] = g_coord(e->g, m, j);
    const double u1 = g_u01(g_hash3(e->g->seed, 101, j)), u2 = g_u01(g_hash3(e->g->seed, 102, j));
    float v;
    if (e->val_dist == 1) {
      const double z = sqrt(-2.0 * log(u1)) * cos(6.283185307179586 * u2);
      v = (float)exp(z);
    } else if (e->val_dist == 2) {
      v = (float)(1 + (int)(u1 * 50.0 < 50.0 ? u1 * 50.0 : 49.0));
    } else {
      v = (float)fma(-u1, 1.0 - 1e-7, 1.0); /* the device contracts 1 - u1 * c into one fused multiply-add */
    }
    e->vals[x] = v;
  }
  return NULL;
}

/* Generate into caller arrays inds[m][nnz] (uint32) and vals[nnz].
 * dist[m]: 0 uniform, 1 Zipf(zipf_s[m]); val_dist: 0 uniform (0,1],
 * 1 lognormal(0,1), 2 integers 1..50. Returns 0, or -1 on bad arguments /
 * allocation failure, -2 when the candidate counter would overflow. */
int orc_generate(int nd, const u64* dims, u64 nnz, const int* dist, const double* zipf_s, int val_dist, u64 seed,
                 int threads, u32** inds, float* vals) {
  if (nd < 3 || nd > 4 || !dims || !dist || !inds || !vals) return -1;
  const int T = threads > 0 ? (threads > 256 ? 256 : threads) : 1;
  gen_t g;
  memset(&g, 0, sizeof(g));
  g.nd = nd;
  g.seed = seed;
  u64 mult = 1;
  for (int m = nd - 1; m >= 0; --m) {
    g.radix[m] = mult;
    mult *= dims[m];
  }
  int rc = 0;
  for (int m = 0; m < nd; ++m) {
    const u64 d = dims[m];
    g.dims[m] = d;
    g.dist[m] = dist[m];
    if (dist[m] == 1) { /* the same CDF and permutation as the library's host set-up */
      const double sx = zipf_s[m];
      g.cdf[m] = (double*)malloc(d * sizeof(double));
      g.perm[m] = (u32*)malloc(d * sizeof(u32));
      if (!g.cdf[m] || !g.perm[m]) { rc = -1; goto done; }
      double acc = 0;
      for (u64 k = 0; k < d; ++k) {
        acc += pow((double)(k + 1), -sx);
        g.cdf[m][k] = acc;
      }
      for (u64 k = 0; k < d; ++k) g.cdf[m][k] /= acc;
      g.cdf[m][d - 1] = 1.0;
      for (u64 k = 0; k < d; ++k) g.perm[m][k] = (u32)k;
      u64 st = g_splitmix(seed ^ (0xabcdef12345ull + (u64)m));
      for (u64 k = d - 1; k > 0; --k) {
        st = g_splitmix(st);
        const u64 r = st % (k + 1);
        const u32 t = g.perm[m][k];
        g.perm[m][k] = g.perm[m][r];
        g.perm[m][r] = t;
      }
    }
  }
  {
    u64* tab[256];
    u64 cap[256], fill[256];
    const u64 per = (nnz + nnz / 4 + 1024) / (u64)T + 1024;
    u64 c0 = 1024;
    while (c0 < per * 2) c0 <<= 1;
    for (int t = 0; t < T; ++t) {
      cap[t] = c0;
      fill[t] = 0;
      tab[t] = (u64*)malloc(c0 * sizeof(u64));
      if (!tab[t]) {
        for (int u = 0; u < t; ++u) free(tab[u]);
        rc = -1;
        goto done;
      }
      memset(tab[t], 0xff, c0 * sizeof(u64));
    }
    u64* cand = (u64*)malloc((nnz ? nnz : 1) * sizeof(u64)); /* kept candidates, j ascending */
    u64 kept = 0, next = 0;
    pthread_t th[256];
    work_t w[256];
    while (kept < nnz && rc == 0) {
      const u64 need = nnz - kept, draw = need + need / 4 + 1024;
      if (next + draw >= (1ull << 32)) { rc = -2; break; } /* the device's counter is 32-bit */
      u64* keys = (u64*)malloc(draw * sizeof(u64));
      unsigned char* kf = (unsigned char*)calloc(draw, 1);
      if (!cand || !keys || !kf) { free(keys); free(kf); rc = -1; break; }
      for (int t = 0; t < T; ++t) {
        w[t] = (work_t){&g, next, draw, keys, kf, t, T, tab, cap, fill, 0};
        pthread_create(&th[t], NULL, g_keys_thread, &w[t]);
      }
      for (int t = 0; t < T; ++t) pthread_join(th[t], NULL);
      for (int t = 0; t < T; ++t) pthread_create(&th[t], NULL, g_dedup_thread, &w[t]);
      for (int t = 0; t < T; ++t) pthread_join(th[t], NULL);
      for (int t = 0; t < T; ++t)
        if (w[t].fail) rc = -1;
      for (u64 i = 0; i < draw && kept < nnz && rc == 0; ++i)
        if (kf[i]) cand[kept++] = next + i;
      next += draw;
      free(keys);
      free(kf);
    }
    for (int t = 0; t < T; ++t) free(tab[t]);
    if (rc == 0 && nnz) {
      emit_t e[256];
      for (int t = 0; t < T; ++t) {
        e[t] = (emit_t){&g, cand, nnz, val_dist, inds, vals, t, T};
        pthread_create(&th[t], NULL, g_emit_thread, &e[t]);
      }
      for (int t = 0; t < T; ++t) pthread_join(th[t], NULL);
    }
    free(cand);
  }
done:
  for (int m = 0; m < 4; ++m) {
    free(g.cdf[m]);
    free(g.perm[m]);
  }
  return rc;
}
