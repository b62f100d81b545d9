/*
 * CPU ORACLE -- test infrastructure only, never part of the product path.
 *
 * A plain-C restatement of the reference's direct J/K driver, linked against
 * the reference's own vendored libcint 6.1.3 (compiled from source into
 * oracle/_ref/libcint_ref.so by oracle/Makefile).  Only tests/, the smoke
 * check and bench.py's CPU-baseline leg load this library.
 *
 * Reference files restated here (paths inside src/gradscf/integrals/_native/):
 *   csrc/tables.h:31-76            table validation, AO offsets
 *   csrc/coulomb_shells.h:10       pair_index
 *   csrc/coulomb_shells.h:60-77    eri_schwarz_bounds
 *   csrc/coulomb_shells.h:80-128   unique_eri traversal (pair pre-skip, AO dedupe)
 *   csrc/direct_jk.cc:7-95         worker row ownership + J/K digestion
 *   csrc/eri_geometry_entries.h:6-31   int2e_ip1 entries, four permutations
 *   csrc/direct_jk_geometry.cc:68-84   transposed (VJP) contraction
 *   csrc/direct_jk_geometry.cc:122-176 per-worker partial + fixed-order reduction
 *   csrc/direct_jk_geometry.cc:8-99    geometry JVP (order 1, 2) and order-2 VJP
 *   csrc/geometry_contraction.h:7-53   second-derivative ERI entries (ipip1, ipvip1, ip1ip2)
 * Workers are pthreads instead of XLA's pool; the partition of output
 * rows (direct J/K) and first shells (geometry VJP) is the reference's, so the
 * arithmetic order within each output element is the reference's too.
 */
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <pthread.h>
#include <unistd.h>

typedef struct CINTOpt CINTOpt;
typedef int (*intor_t)(double *, int *, int *, int *, int, int *, int, double *,
                       CINTOpt *, double *);
extern int int2e_sph(double *, int *, int *, int *, int, int *, int, double *, CINTOpt *, double *);
extern int int2e_cart(double *, int *, int *, int *, int, int *, int, double *, CINTOpt *, double *);
extern int int2e_ip1_sph(double *, int *, int *, int *, int, int *, int, double *, CINTOpt *, double *);
extern int int2e_ip1_cart(double *, int *, int *, int *, int, int *, int, double *, CINTOpt *, double *);
extern int int2e_ipip1_sph(double *, int *, int *, int *, int, int *, int, double *, CINTOpt *, double *);
extern int int2e_ipip1_cart(double *, int *, int *, int *, int, int *, int, double *, CINTOpt *, double *);
extern int int2e_ipvip1_sph(double *, int *, int *, int *, int, int *, int, double *, CINTOpt *, double *);
extern int int2e_ipvip1_cart(double *, int *, int *, int *, int, int *, int, double *, CINTOpt *, double *);
extern int int2e_ip1ip2_sph(double *, int *, int *, int *, int, int *, int, double *, CINTOpt *, double *);
extern int int2e_ip1ip2_cart(double *, int *, int *, int *, int, int *, int, double *, CINTOpt *, double *);
extern void int2e_optimizer(CINTOpt **, int *, int, int *, int, double *);
extern void CINTdel_optimizer(CINTOpt **);
extern int int1e_ovlp_sph(double *, int *, int *, int *, int, int *, int, double *, CINTOpt *, double *);
extern int int1e_ovlp_cart(double *, int *, int *, int *, int, int *, int, double *, CINTOpt *, double *);
extern int int1e_kin_sph(double *, int *, int *, int *, int, int *, int, double *, CINTOpt *, double *);
extern int int1e_kin_cart(double *, int *, int *, int *, int, int *, int, double *, CINTOpt *, double *);
extern int int1e_nuc_sph(double *, int *, int *, int *, int, int *, int, double *, CINTOpt *, double *);
extern int int1e_nuc_cart(double *, int *, int *, int *, int, int *, int, double *, CINTOpt *, double *);
extern int int1e_ipovlp_sph(double *, int *, int *, int *, int, int *, int, double *, CINTOpt *, double *);
extern int int1e_ipovlp_cart(double *, int *, int *, int *, int, int *, int, double *, CINTOpt *, double *);
extern int int1e_ipkin_sph(double *, int *, int *, int *, int, int *, int, double *, CINTOpt *, double *);
extern int int1e_ipkin_cart(double *, int *, int *, int *, int, int *, int, double *, CINTOpt *, double *);
extern int int1e_ipnuc_sph(double *, int *, int *, int *, int, int *, int, double *, CINTOpt *, double *);
extern int int1e_ipnuc_cart(double *, int *, int *, int *, int, int *, int, double *, CINTOpt *, double *);
extern int int1e_iprinv_sph(double *, int *, int *, int *, int, int *, int, double *, CINTOpt *, double *);
extern int int1e_iprinv_cart(double *, int *, int *, int *, int, int *, int, double *, CINTOpt *, double *);

/* libcint slot layout (cint.h) */
enum { ATM_SLOTS = 6, BAS_SLOTS = 8, PTR_ENV_START = 20, PTR_RINV_ORIG = 4,
       PTR_RANGE_OMEGA = 8, CHARGE_OF = 0, PTR_COORD = 1, NUC_MOD_OF = 2,
       ATOM_OF = 0, ANG_OF = 1, NPRIM_OF = 2, NCTR_OF = 3, KAPPA_OF = 4,
       PTR_EXP = 5, PTR_COEFF = 6 };

static __thread char g_err[512];
const char *oracle_last_error(void) { return g_err; }
static int fail(const char *msg) {
  snprintf(g_err, sizeof g_err, "%s", msg);
  return 1;
}

typedef struct {
  int natm, nbas, n, nenv;
  int *atm, *bas, *ao;
  double *env;
} tables_t;

/* tables.h:31-76 -- copy + validate; AO offsets ao[s+1] = ao[s] + nctr*dim(l). */
static int tables_init(tables_t *t, const int32_t *atm, int natm, const int32_t *bas,
                       int nbas, const double *env, int nenv, int cart) {
  memset(t, 0, sizeof *t);
  if (nenv < 20 || (cart != 0 && cart != 1) || natm < 0 || nbas < 1)
    return fail("Invalid libcint table dimensions or operator");
  t->natm = natm; t->nbas = nbas; t->nenv = nenv;
  t->atm = malloc(sizeof(int) * (size_t)natm * ATM_SLOTS + 1);
  t->bas = malloc(sizeof(int) * (size_t)nbas * BAS_SLOTS);
  t->env = malloc(sizeof(double) * (size_t)nenv);
  t->ao = malloc(sizeof(int) * (size_t)(nbas + 1));
  memcpy(t->atm, atm, sizeof(int) * (size_t)natm * ATM_SLOTS);
  memcpy(t->bas, bas, sizeof(int) * (size_t)nbas * BAS_SLOTS);
  memcpy(t->env, env, sizeof(double) * (size_t)nenv);
  for (int i = 0; i < nenv; ++i)
    if (!isfinite(t->env[i])) return fail("Native integral env must be finite");
  if (t->env[PTR_RANGE_OMEGA] < 0.) return fail("omega must be nonnegative");
  for (int a = 0; a < natm; ++a) {
    const int *row = t->atm + a * ATM_SLOTS;
    if (row[PTR_COORD] < PTR_ENV_START || row[PTR_COORD] + 3 > nenv || row[NUC_MOD_OF] != 1)
      return fail("Native backend requires valid point nuclei");
  }
  t->ao[0] = 0;
  for (int s = 0; s < nbas; ++s) {
    const int *row = t->bas + s * BAS_SLOTS;
    int l = row[ANG_OF], np = row[NPRIM_OF], nc = row[NCTR_OF];
    if (row[ATOM_OF] < 0 || row[ATOM_OF] >= natm || l < 0 || l > 12 || np < 1 || np > 64 ||
        nc < 1 || nc > 64 || row[KAPPA_OF] != 0 || row[PTR_EXP] < PTR_ENV_START ||
        row[PTR_EXP] + np > nenv || row[PTR_COEFF] < PTR_ENV_START ||
        (int64_t)row[PTR_COEFF] + (int64_t)np * nc > nenv)
      return fail("Invalid or unsupported libcint basis table");
    for (int p = 0; p < np; ++p)
      if (t->env[row[PTR_EXP] + p] <= 0.) return fail("Gaussian exponents must be positive");
    t->ao[s + 1] = t->ao[s] + nc * (cart ? (l + 1) * (l + 2) / 2 : 2 * l + 1);
  }
  t->n = t->ao[nbas];
  if (t->n < 1) return fail("Invalid AO count");
  return 0;
}

static void tables_free(tables_t *t) {
  free(t->atm); free(t->bas); free(t->env); free(t->ao);
}

/* coulomb_shells.h:10 */
static size_t pair_index(size_t a, size_t b) {
  if (a < b) { size_t t = a; a = b; b = t; }
  return a * (a + 1) / 2 + b;
}

typedef struct { double *data; size_t cap; double *cache; size_t ccap; } scratch_t;

/* coulomb_shells.h:32-58 -- zero the block, then one libcint call. */
static void eval_block(tables_t *t, intor_t f, CINTOpt *opt, int *sh, size_t count,
                       scratch_t *s) {
  if (count > s->cap) { free(s->data); s->data = malloc(count * sizeof(double)); s->cap = count; }
  int length = f(NULL, NULL, sh, t->atm, t->natm, t->bas, t->nbas, t->env, opt, NULL);
  if ((size_t)length > s->ccap) {
    free(s->cache); s->cache = malloc((size_t)length * sizeof(double)); s->ccap = (size_t)length;
  }
  memset(s->data, 0, count * sizeof(double));
  f(s->data, NULL, sh, t->atm, t->natm, t->bas, t->nbas, t->env, opt, s->cache);
}

/* coulomb_shells.h:60-77 -- Q_ij = sqrt(max_pq |(pq|pq)|), only j <= i stored. */
static int schwarz_bounds(tables_t *t, int cart, double cutoff, CINTOpt *opt, double *bounds) {
  if (!isfinite(cutoff) || cutoff < 0) return fail("Invalid Schwarz cutoff");
  intor_t f = cart ? int2e_cart : int2e_sph;
  scratch_t s = {0};
  memset(bounds, 0, sizeof(double) * (size_t)t->nbas * t->nbas);
  for (int i = 0; i < t->nbas; ++i)
    for (int j = 0; j <= i; ++j) {
      int sh[4] = {i, j, i, j};
      int di = t->ao[i + 1] - t->ao[i], dj = t->ao[j + 1] - t->ao[j];
      eval_block(t, f, opt, sh, (size_t)di * dj * di * dj, &s);
      double largest = 0.;
      for (int p = 0; p < di; ++p)
        for (int q = 0; q < dj; ++q) {
          double v = fabs(s.data[(((size_t)q * di + p) * dj + q) * di + p]);
          if (v > largest) largest = v;
        }
      bounds[(size_t)i * t->nbas + j] = sqrt(largest);
    }
  free(s.data); free(s.cache);
  return 0;
}

int oracle_schwarz_bounds(const int32_t *atm, int natm, const int32_t *bas, int nbas,
                          const double *env, int nenv, int cart, double *bounds) {
  tables_t t;
  if (tables_init(&t, atm, natm, bas, nbas, env, nenv, cart)) { tables_free(&t); return 1; }
  CINTOpt *opt = NULL;
  int2e_optimizer(&opt, t.atm, t.natm, t.bas, t.nbas, t.env);
  int rc = schwarz_bounds(&t, cart, 1.0, opt, bounds);
  CINTdel_optimizer(&opt);
  tables_free(&t);
  return rc;
}

/* direct_jk.cc:45-77 digestion for one unique AO integral, restricted to the
 * worker's owned rows [row_begin,row_end). */
static inline void digest(int a, int b, int c, int e, double v, int n, int nb,
                          const double *d, double *out, int with_j, int with_k,
                          int row_begin, int row_end) {
  const size_t nn = (size_t)n * n;
  const size_t ab = pair_index(a, b), ce = pair_index(c, e);
#define OWNS(r) (row_begin <= (r) && (r) < row_end)
  const int own_a = OWNS(a), own_b = OWNS(b), own_c = OWNS(c), own_e = OWNS(e);
#undef OWNS
  for (int batch = 0; batch < nb; ++batch) {
    const double *dm = d + (size_t)batch * nn;
    if (with_j) {
      double *j = out + (size_t)batch * nn;
      if (own_a || own_b) {
        double j_ab = v * (dm[(size_t)c * n + e] + (c != e ? dm[(size_t)e * n + c] : 0.));
        if (own_a) j[(size_t)a * n + b] += j_ab;
        if (a != b && own_b) j[(size_t)b * n + a] += j_ab;
      }
      if (ab != ce && (own_c || own_e)) {
        double j_ce = v * (dm[(size_t)a * n + b] + (a != b ? dm[(size_t)b * n + a] : 0.));
        if (own_c) j[(size_t)c * n + e] += j_ce;
        if (c != e && own_e) j[(size_t)e * n + c] += j_ce;
      }
    }
    if (with_k) {
      double *k = out + (size_t)(with_j * nb + batch) * nn;
      if (own_a) k[(size_t)a * n + c] += v * dm[(size_t)b * n + e];
      if (c != e && own_a) k[(size_t)a * n + e] += v * dm[(size_t)b * n + c];
      if (a != b && own_b) k[(size_t)b * n + c] += v * dm[(size_t)a * n + e];
      if (a != b && c != e && own_b) k[(size_t)b * n + e] += v * dm[(size_t)a * n + c];
      if (ab != ce) {
        if (own_c) k[(size_t)c * n + a] += v * dm[(size_t)e * n + b];
        if (a != b && own_c) k[(size_t)c * n + b] += v * dm[(size_t)e * n + a];
        if (c != e && own_e) k[(size_t)e * n + a] += v * dm[(size_t)c * n + b];
        if (a != b && c != e && own_e) k[(size_t)e * n + b] += v * dm[(size_t)c * n + a];
      }
    }
  }
}

/* coulomb_shells.h:80-128 -- the unique_eri traversal for one worker's shell
 * range [sb,se).  Returns the number of libcint shell-quartet calls made. */
static long long unique_eri_worker(tables_t *t, int cart, double cutoff, int sb, int se,
                                   const double *bounds, double largest, CINTOpt *opt,
                                   int nb, const double *d, double *out, int with_j,
                                   int with_k) {
  intor_t f = cart ? int2e_cart : int2e_sph;
  scratch_t s = {0};
  long long calls = 0;
  const int row_begin = t->ao[sb], row_end = t->ao[se];
#define OWNSH(x) (sb <= (x) && (x) < se)
  for (int i = sb; i < t->nbas; ++i)
    for (int j = 0; j <= i; ++j) {
      if (cutoff > 0 && bounds[(size_t)i * t->nbas + j] * largest < cutoff) continue;
      const int outer_owned = OWNSH(i) || OWNSH(j);
      for (int k = outer_owned ? 0 : sb; k <= i; ++k) {
        const int owned = outer_owned || OWNSH(k);
        const int first = owned ? 0 : sb;
        const int last = owned ? k + 1 : (k + 1 < se ? k + 1 : se);
        for (int l = first; l < last; ++l) {
          if (cutoff > 0 &&
              bounds[(size_t)i * t->nbas + j] * bounds[(size_t)k * t->nbas + l] < cutoff)
            continue;
          const int di = t->ao[i + 1] - t->ao[i], dj = t->ao[j + 1] - t->ao[j];
          const int dk = t->ao[k + 1] - t->ao[k], dl = t->ao[l + 1] - t->ao[l];
          int sh[4] = {i, j, k, l};
          eval_block(t, f, opt, sh, (size_t)di * dj * dk * dl, &s);
          ++calls;
          for (int p = 0; p < di; ++p)
            for (int q = 0; q < dj; ++q) {
              const int a = t->ao[i] + p, b = t->ao[j] + q;
              if (a < b) continue;
              const size_t ab = pair_index(a, b);
              for (int r = 0; r < dk; ++r)
                for (int w = 0; w < dl; ++w) {
                  const int c = t->ao[k] + r, e = t->ao[l] + w;
                  if (c < e || ab < pair_index(c, e)) continue;
                  digest(a, b, c, e, s.data[(((size_t)w * dk + r) * dj + q) * di + p], t->n, nb,
                         d, out, with_j, with_k, row_begin, row_end);
                }
            }
        }
      }
    }
#undef OWNSH
  free(s.data); free(s.cache);
  return calls;
}

static int host_threads(void) {
  long c = sysconf(_SC_NPROCESSORS_ONLN);
  return c > 0 ? (int)c : 1;
}

typedef struct {
  tables_t *t; int cart; double cutoff; int sb, se; const double *bounds; double largest;
  CINTOpt *opt; int nb; const double *d; double *out; int with_j, with_k; long long calls;
} jk_task_t;

static void *jk_task_run(void *arg) {
  jk_task_t *k = (jk_task_t *)arg;
  k->calls = unique_eri_worker(k->t, k->cart, k->cutoff, k->sb, k->se, k->bounds, k->largest,
                               k->opt, k->nb, k->d, k->out, k->with_j, k->with_k);
  return NULL;
}

/* direct_jk.cc:7-95.  out has shape (with_j+with_k, nb, n, n); it is fully
 * overwritten.  Returns 0 on success, nonzero with oracle_last_error(). */
int oracle_direct_jk(const int32_t *atm, int natm, const int32_t *bas, int nbas,
                     const double *env, int nenv, const double *density, int nb, int n,
                     double *out, int cart, double cutoff, int workers, int with_j,
                     int with_k, long long *calls_out) {
  if (workers < 1) return fail("Direct J/K workers must be positive");
  if ((with_j != 0 && with_j != 1) || (with_k != 0 && with_k != 1) || !(with_j || with_k))
    return fail("Direct J/K requires at least one selected operator");
  tables_t t;
  if (tables_init(&t, atm, natm, bas, nbas, env, nenv, cart)) { tables_free(&t); return 1; }
  if (n != t.n) { tables_free(&t); return fail("Direct J/K shape mismatch"); }
  for (size_t i = 0; i < (size_t)nb * n * n; ++i)
    if (!isfinite(density[i])) { tables_free(&t); return fail("Nonfinite density"); }
  if (!isfinite(cutoff) || cutoff < 0) { tables_free(&t); return fail("Invalid Schwarz cutoff"); }
  int w = workers < host_threads() ? workers : host_threads();
  if (w > t.nbas) w = t.nbas;
  if (w < 1) w = 1;
  memset(out, 0, sizeof(double) * (size_t)(with_j + with_k) * nb * n * n);
  CINTOpt *opt = NULL;
  int2e_optimizer(&opt, t.atm, t.natm, t.bas, t.nbas, t.env);
  double *bounds = NULL, largest = 0.;
  if (cutoff > 0) {
    bounds = malloc(sizeof(double) * (size_t)t.nbas * t.nbas);
    schwarz_bounds(&t, cart, cutoff, opt, bounds);
    for (size_t i = 0; i < (size_t)t.nbas * t.nbas; ++i) if (bounds[i] > largest) largest = bounds[i];
  }
  jk_task_t *tasks = calloc((size_t)w, sizeof(jk_task_t));
  pthread_t *threads = calloc((size_t)w, sizeof(pthread_t));
  for (int worker = 0; worker < w; ++worker) {
    jk_task_t task = {&t, cart, cutoff, worker * t.nbas / w, (worker + 1) * t.nbas / w, bounds,
                      largest, opt, nb, density, out, with_j, with_k, 0};
    tasks[worker] = task;
  }
  for (int worker = 1; worker < w; ++worker) pthread_create(&threads[worker], NULL, jk_task_run, &tasks[worker]);
  jk_task_run(&tasks[0]);
  for (int worker = 1; worker < w; ++worker) pthread_join(threads[worker], NULL);
  long long calls = 0;
  for (int worker = 0; worker < w; ++worker) calls += tasks[worker].calls;
  free(tasks); free(threads);
  if (calls_out) *calls_out = calls;
  free(bounds);
  CINTdel_optimizer(&opt);
  tables_free(&t);
  return 0;
}

/* Full s1 ERI tensor (n^4), the einsum oracle of the reference's tests
 * (tests/integrals/test_native_direct_parallel.py:45-50): out[((p*n+q)*n+r)*n+s]. */
int oracle_eri_s1(const int32_t *atm, int natm, const int32_t *bas, int nbas, const double *env,
                  int nenv, int cart, double *out) {
  tables_t t;
  if (tables_init(&t, atm, natm, bas, nbas, env, nenv, cart)) { tables_free(&t); return 1; }
  const size_t n = t.n;
  intor_t f = cart ? int2e_cart : int2e_sph;
  CINTOpt *opt = NULL;
  int2e_optimizer(&opt, t.atm, t.natm, t.bas, t.nbas, t.env);
  {
    scratch_t s = {0};
    for (int i = 0; i < t.nbas; ++i)
      for (int j = 0; j < t.nbas; ++j)
        for (int k = 0; k < t.nbas; ++k)
          for (int l = 0; l < t.nbas; ++l) {
            int sh[4] = {i, j, k, l};
            int di = t.ao[i + 1] - t.ao[i], dj = t.ao[j + 1] - t.ao[j];
            int dk = t.ao[k + 1] - t.ao[k], dl = t.ao[l + 1] - t.ao[l];
            eval_block(&t, f, opt, sh, (size_t)di * dj * dk * dl, &s);
            for (int w = 0; w < dl; ++w)
              for (int r = 0; r < dk; ++r)
                for (int q = 0; q < dj; ++q)
                  for (int p = 0; p < di; ++p)
                    out[(((size_t)(t.ao[i] + p) * n + t.ao[j] + q) * n + t.ao[k] + r) * n +
                        t.ao[l] + w] = s.data[(((size_t)w * dk + r) * dj + q) * di + p];
          }
    free(s.data); free(s.cache);
  }
  CINTdel_optimizer(&opt);
  tables_free(&t);
  return 0;
}

/* One shell quartet block in libcint's layout (first index fastest), for
 * element-wise kernel checks: out[((s*dk+r)*dj+q)*di+p]. */
int oracle_eri_block(const int32_t *atm, int natm, const int32_t *bas, int nbas,
                     const double *env, int nenv, int cart, const int32_t *shls, double *out) {
  tables_t t;
  if (tables_init(&t, atm, natm, bas, nbas, env, nenv, cart)) { tables_free(&t); return 1; }
  int sh[4] = {shls[0], shls[1], shls[2], shls[3]};
  scratch_t s = {0};
  size_t count = 1;
  for (int a = 0; a < 4; ++a) count *= (size_t)(t.ao[sh[a] + 1] - t.ao[sh[a]]);
  eval_block(&t, cart ? int2e_cart : int2e_sph, NULL, sh, count, &s);
  memcpy(out, s.data, count * sizeof(double));
  free(s.data); free(s.cache);
  tables_free(&t);
  return 0;
}

/* One-electron matrices: which = 0 overlap, 1 kinetic, 2 nuclear attraction
 * (all atoms with their charges; zero-charge basis centres add nothing). */
int oracle_int1e(const int32_t *atm, int natm, const int32_t *bas, int nbas, const double *env,
                 int nenv, int cart, int which, double *out) {
  tables_t t;
  if (tables_init(&t, atm, natm, bas, nbas, env, nenv, cart)) { tables_free(&t); return 1; }
  intor_t table[3][2] = {{int1e_ovlp_sph, int1e_ovlp_cart}, {int1e_kin_sph, int1e_kin_cart},
                         {int1e_nuc_sph, int1e_nuc_cart}};
  if (which < 0 || which > 2) { tables_free(&t); return fail("bad operator"); }
  intor_t f = table[which][cart];
  const size_t n = t.n;
  scratch_t s = {0};
  for (int i = 0; i < t.nbas; ++i)
    for (int j = 0; j < t.nbas; ++j) {
      int sh[4] = {i, j, 0, 0};
      int di = t.ao[i + 1] - t.ao[i], dj = t.ao[j + 1] - t.ao[j];
      eval_block(&t, f, NULL, sh, (size_t)di * dj, &s);
      for (int q = 0; q < dj; ++q)
        for (int p = 0; p < di; ++p)
          out[(size_t)(t.ao[i] + p) * n + t.ao[j] + q] = s.data[(size_t)q * di + p];
    }
  free(s.data); free(s.cache);
  tables_free(&t);
  return 0;
}

/* Bra-centre derivative one-electron blocks, libcint sign convention
 * (d/d r of the bra function, i.e. minus the centre derivative):
 * which = 0 ipovlp, 1 ipkin, 2 ipnuc, 3 iprinv about atom `rinv_atom`.
 * out has shape (3, n, n). */
int oracle_int1e_ip(const int32_t *atm, int natm, const int32_t *bas, int nbas,
                    const double *env, int nenv, int cart, int which, int rinv_atom,
                    double *out) {
  tables_t t;
  if (tables_init(&t, atm, natm, bas, nbas, env, nenv, cart)) { tables_free(&t); return 1; }
  intor_t table[4][2] = {{int1e_ipovlp_sph, int1e_ipovlp_cart}, {int1e_ipkin_sph, int1e_ipkin_cart},
                         {int1e_ipnuc_sph, int1e_ipnuc_cart}, {int1e_iprinv_sph, int1e_iprinv_cart}};
  if (which < 0 || which > 3) { tables_free(&t); return fail("bad operator"); }
  if (which == 3) {
    if (rinv_atom < 0 || rinv_atom >= t.natm) { tables_free(&t); return fail("bad atom"); }
    const double *r = t.env + t.atm[rinv_atom * ATM_SLOTS + PTR_COORD];
    t.env[PTR_RINV_ORIG] = r[0]; t.env[PTR_RINV_ORIG + 1] = r[1]; t.env[PTR_RINV_ORIG + 2] = r[2];
  }
  intor_t f = table[which][cart];
  const size_t n = t.n;
  scratch_t s = {0};
  for (int i = 0; i < t.nbas; ++i)
    for (int j = 0; j < t.nbas; ++j) {
      int sh[4] = {i, j, 0, 0};
      int di = t.ao[i + 1] - t.ao[i], dj = t.ao[j + 1] - t.ao[j];
      const size_t sz = (size_t)di * dj;
      eval_block(&t, f, NULL, sh, 3 * sz, &s);
      for (int x = 0; x < 3; ++x)
        for (int q = 0; q < dj; ++q)
          for (int p = 0; p < di; ++p)
            out[(size_t)x * n * n + (size_t)(t.ao[i] + p) * n + t.ao[j] + q] =
                s.data[x * sz + (size_t)q * di + p];
    }
  free(s.data); free(s.cache);
  tables_free(&t);
  return 0;
}

/* direct_jk_geometry.cc:68-84 (transpose=true, order 1) over
 * eri_geometry_entries.h:6-31 entries, for first shells [fs,ls). */
static void geometry_vjp_range(tables_t *t, int cart, int nb, const double *dm, const double *input,
                               int with_j, int with_k, int fs, int ls, double *output) {
  const int n = t->n;
  const size_t nn = (size_t)n * n;
  intor_t ip = cart ? int2e_ip1_cart : int2e_ip1_sph;
  scratch_t s = {0};
  for (int i = fs; i < ls; ++i)
    for (int j = 0; j < t->nbas; ++j)
      for (int k = 0; k < t->nbas; ++k)
        for (int l = 0; l < t->nbas; ++l) {
          int sh[4] = {i, j, k, l};
          const int di = t->ao[i + 1] - t->ao[i], dj = t->ao[j + 1] - t->ao[j];
          const int dk = t->ao[k + 1] - t->ao[k], dl = t->ao[l + 1] - t->ao[l];
          const size_t size = (size_t)di * dj * dk * dl;
          eval_block(t, ip, NULL, sh, 3 * size, &s);
          const int coord0 = t->atm[t->bas[i * BAS_SLOTS + ATOM_OF] * ATM_SLOTS + PTR_COORD];
          for (int x = 0; x < 3; ++x)
            for (int w = 0; w < dl; ++w)
              for (int r = 0; r < dk; ++r)
                for (int q = 0; q < dj; ++q)
                  for (int p = 0; p < di; ++p) {
                    const double value = -s.data[x * size + (((size_t)w * dk + r) * dj + q) * di + p];
                    const int a = t->ao[i] + p, b = t->ao[j] + q, c = t->ao[k] + r, d = t->ao[l] + w;
                    const int perm[4][4] = {{a, b, c, d}, {b, a, c, d}, {c, d, a, b}, {c, d, b, a}};
                    for (int e = 0; e < 4; ++e) {
                      const int A = perm[e][0], B = perm[e][1], C = perm[e][2], D = perm[e][3];
                      double sum = 0.;
                      for (int batch = 0; batch < nb; ++batch) {
                        const double *dmat = dm + (size_t)batch * nn;
                        if (with_j) sum += input[(size_t)batch * nn + (size_t)A * n + B] * dmat[(size_t)C * n + D];
                        if (with_k)
                          sum += input[(size_t)(with_j * nb + batch) * nn + (size_t)A * n + C] *
                                 dmat[(size_t)B * n + D];
                      }
                      output[coord0 + x] += value * sum;
                    }
                  }
        }
  free(s.data); free(s.cache);
}

typedef struct {
  const int32_t *atm; int natm; const int32_t *bas; int nbas; const double *env; int nenv;
  int cart, nb; const double *dm, *input; int with_j, with_k, fs, ls; double *output;
} vjp_task_t;

static void *vjp_task_run(void *arg) {
  vjp_task_t *k = (vjp_task_t *)arg;
  tables_t local;
  tables_init(&local, k->atm, k->natm, k->bas, k->nbas, k->env, k->nenv, k->cart);
  geometry_vjp_range(&local, k->cart, k->nb, k->dm, k->input, k->with_j, k->with_k, k->fs, k->ls,
                     k->output);
  tables_free(&local);
  return NULL;
}

/* direct_jk_geometry.cc:122-182: coordinate VJP of J/K.  vector (the J/K
 * cotangent) has shape (with_j+with_k, nb, n, n); out is env-sized and is
 * fully overwritten.  Per-worker partials are summed in worker order. */
int oracle_direct_jk_geometry_vjp(const int32_t *atm, int natm, const int32_t *bas, int nbas,
                                  const double *env, int nenv, const double *density, int nb,
                                  int n, const double *vector, double *out, int cart, int with_j,
                                  int with_k, int workers) {
  if (workers < 1) return fail("Direct J/K geometry workers must be positive");
  if ((with_j != 0 && with_j != 1) || (with_k != 0 && with_k != 1) || !(with_j || with_k))
    return fail("Invalid direct J/K geometry product");
  tables_t t;
  if (tables_init(&t, atm, natm, bas, nbas, env, nenv, cart)) { tables_free(&t); return 1; }
  if (n != t.n) { tables_free(&t); return fail("Direct J/K geometry density shape mismatch"); }
  int w = workers < host_threads() ? workers : host_threads();
  if (w > t.nbas) w = t.nbas;
  double *partials = calloc((size_t)w * nenv, sizeof(double));
  vjp_task_t *tasks = calloc((size_t)w, sizeof(vjp_task_t));
  pthread_t *threads = calloc((size_t)w, sizeof(pthread_t));
  for (int worker = 0; worker < w; ++worker) {
    vjp_task_t task = {atm, natm, bas, nbas, env, nenv, cart, nb, density, vector, with_j, with_k,
                       worker * t.nbas / w, (worker + 1) * t.nbas / w,
                       partials + (size_t)worker * nenv};
    tasks[worker] = task;
  }
  for (int worker = 1; worker < w; ++worker) pthread_create(&threads[worker], NULL, vjp_task_run, &tasks[worker]);
  vjp_task_run(&tasks[0]);
  for (int worker = 1; worker < w; ++worker) pthread_join(threads[worker], NULL);
  free(tasks); free(threads);
  memset(out, 0, sizeof(double) * (size_t)nenv);
  for (int worker = 0; worker < w; ++worker)
    for (int i = 0; i < nenv; ++i) out[i] += partials[(size_t)worker * nenv + i];
  free(partials);
  tables_free(&t);
  return 0;
}

/* ---------------------------------------------------------------------------
 * Geometry products of J/K (direct_jk_geometry.cc:8-99).
 *   transpose = 0 (JVP): out (with_j+with_k, nb, n, n) = d/du J/K (order 1) or
 *     d^2/du dv J/K (order 2); u = direction, v = vector (env-sized).
 *   transpose = 1 (order-2 VJP): out (env-sized) = the coordinate gradient of
 *     sum(Jbar * dJ/du + Kbar * dK/du); vector = (Jbar, Kbar) cotangents.
 * Every ordered shell quartet (eri_window.h:91-105 without a window), per
 * worker a range of first shells, partials summed in worker order. */
typedef struct {
  tables_t *t; int n, nb, with_j, with_k, transpose;
  const double *dm, *u, *input; double *output;
} geo_ctx_t;

/* direct_jk_geometry.cc:65-81, the consume lambda */
static void geo_consume(geo_ctx_t *g, int a, int b, int c, int d, int coordinate, double value) {
  const int n = g->n;
  const size_t nn = (size_t)n * n;
  double sum = 0.;
  for (int batch = 0; batch < g->nb; ++batch) {
    const double *dmat = g->dm + (size_t)batch * nn;
    if (g->transpose) {
      if (g->with_j) sum += g->input[(size_t)batch * nn + (size_t)a * n + b] * dmat[(size_t)c * n + d];
      if (g->with_k)
        sum += g->input[(size_t)(g->with_j * g->nb + batch) * nn + (size_t)a * n + c] * dmat[(size_t)b * n + d];
    } else {
      if (g->with_j) g->output[(size_t)batch * nn + (size_t)a * n + b] += value * dmat[(size_t)c * n + d];
      if (g->with_k)
        g->output[(size_t)(g->with_j * g->nb + batch) * nn + (size_t)a * n + c] += value * dmat[(size_t)b * n + d];
    }
  }
  if (g->transpose) g->output[coordinate] += value * sum;
}

/* direct_jk_geometry.cc:94-99: add(index, a, b, value) of the Hessian entries */
static void geo_add2(geo_ctx_t *g, int a, int b, int c, int d, int pa, int pb, double value) {
  geo_consume(g, a, b, c, d, pa, g->transpose ? value * g->u[pb] : value * g->u[pa] * g->input[pb]);
}
static void geo_cross(geo_ctx_t *g, int a, int b, int c, int d, int pa, int pb, double value) {
  geo_add2(g, a, b, c, d, pa, pb, value);
  geo_add2(g, a, b, c, d, pb, pa, value);
}

static int coord_ptr(const tables_t *t, int shell) {
  return t->atm[t->bas[shell * BAS_SLOTS + ATOM_OF] * ATM_SLOTS + PTR_COORD];
}

/* order 1: eri_geometry_entries.h:6-31 entries, direct_jk_geometry.cc:84-88 */
static void geometry_order1_range(geo_ctx_t *g, int cart, int fs, int ls) {
  tables_t *t = g->t;
  intor_t ip = cart ? int2e_ip1_cart : int2e_ip1_sph;
  scratch_t s = {0};
  for (int i = fs; i < ls; ++i)
    for (int j = 0; j < t->nbas; ++j)
      for (int k = 0; k < t->nbas; ++k)
        for (int l = 0; l < t->nbas; ++l) {
          int sh[4] = {i, j, k, l};
          const int di = t->ao[i + 1] - t->ao[i], dj = t->ao[j + 1] - t->ao[j];
          const int dk = t->ao[k + 1] - t->ao[k], dl = t->ao[l + 1] - t->ao[l];
          const size_t size = (size_t)di * dj * dk * dl;
          eval_block(t, ip, NULL, sh, 3 * size, &s);
          const int coord0 = coord_ptr(t, i);
          for (int x = 0; x < 3; ++x)
            for (int w = 0; w < dl; ++w)
              for (int r = 0; r < dk; ++r)
                for (int q = 0; q < dj; ++q)
                  for (int p = 0; p < di; ++p) {
                    const double value = -s.data[x * size + (((size_t)w * dk + r) * dj + q) * di + p];
                    const int a = t->ao[i] + p, b = t->ao[j] + q, c = t->ao[k] + r, d = t->ao[l] + w;
                    const int perm[4][4] = {{a, b, c, d}, {b, a, c, d}, {c, d, a, b}, {c, d, b, a}};
                    for (int e = 0; e < 4; ++e)
                      geo_consume(g, perm[e][0], perm[e][1], perm[e][2], perm[e][3], coord0 + x,
                                  g->transpose ? value : value * g->u[coord0 + x]);
                  }
        }
  free(s.data); free(s.cache);
}

/* order 2: geometry_contraction.h:24-53 (op == 4) */
static void geometry_order2_range(geo_ctx_t *g, int cart, int fs, int ls) {
  tables_t *t = g->t;
  intor_t kernels[3] = {cart ? int2e_ipip1_cart : int2e_ipip1_sph, cart ? int2e_ipvip1_cart : int2e_ipvip1_sph,
                        cart ? int2e_ip1ip2_cart : int2e_ip1ip2_sph};
  scratch_t s = {0};
  for (int i = fs; i < ls; ++i)
    for (int j = 0; j < t->nbas; ++j)
      for (int k = 0; k < t->nbas; ++k)
        for (int l = 0; l < t->nbas; ++l) {
          int sh[4] = {i, j, k, l};
          const int di = t->ao[i + 1] - t->ao[i], dj = t->ao[j + 1] - t->ao[j];
          const int dk = t->ao[k + 1] - t->ao[k], dl = t->ao[l + 1] - t->ao[l];
          const size_t size = (size_t)di * dj * dk * dl;
          for (int kind = 0; kind < 3; ++kind) {
            eval_block(t, kernels[kind], NULL, sh, 9 * size, &s);
            for (int x = 0; x < 3; ++x)
              for (int y = 0; y < 3; ++y)
                for (int w = 0; w < dl; ++w)
                  for (int r = 0; r < dk; ++r)
                    for (int q = 0; q < dj; ++q)
                      for (int p = 0; p < di; ++p) {
                        const double value = s.data[(x * 3 + y) * size + (((size_t)w * dk + r) * dj + q) * di + p];
                        const int a = t->ao[i] + p, b = t->ao[j] + q, c = t->ao[k] + r, d = t->ao[l] + w;
                        const int px = coord_ptr(t, i) + x;
                        if (kind == 0) {
                          const int py = coord_ptr(t, i) + y;
                          geo_add2(g, a, b, c, d, px, py, value); geo_add2(g, b, a, c, d, px, py, value);
                          geo_add2(g, c, d, a, b, px, py, value); geo_add2(g, c, d, b, a, px, py, value);
                        } else if (kind == 1) {
                          const int py = coord_ptr(t, j) + y;
                          geo_cross(g, a, b, c, d, px, py, value);
                          geo_cross(g, c, d, a, b, px, py, value);
                        } else {
                          const int py = coord_ptr(t, k) + y;
                          geo_cross(g, a, b, c, d, px, py, value); geo_cross(g, b, a, c, d, px, py, value);
                          geo_cross(g, a, b, d, c, px, py, value); geo_cross(g, b, a, d, c, px, py, value);
                        }
                      }
          }
        }
  free(s.data); free(s.cache);
}

typedef struct {
  const int32_t *atm; int natm; const int32_t *bas; int nbas; const double *env; int nenv;
  int cart, order, nb, with_j, with_k, transpose; const double *dm, *u, *input;
  int fs, ls; double *output;
} geo_task_t;

static void *geo_task_run(void *arg) {
  geo_task_t *k = (geo_task_t *)arg;
  tables_t local;
  tables_init(&local, k->atm, k->natm, k->bas, k->nbas, k->env, k->nenv, k->cart);
  geo_ctx_t g = {&local, local.n, k->nb, k->with_j, k->with_k, k->transpose, k->dm, k->u, k->input, k->output};
  if (k->order == 1) geometry_order1_range(&g, k->cart, k->fs, k->ls);
  else geometry_order2_range(&g, k->cart, k->fs, k->ls);
  tables_free(&local);
  return NULL;
}

int oracle_direct_jk_geometry_product(const int32_t *atm, int natm, const int32_t *bas, int nbas,
                                      const double *env, int nenv, const double *density, int nb,
                                      int n, const double *direction, const double *vector,
                                      double *out, int order, int transpose, int cart, int with_j,
                                      int with_k, int workers) {
  if (workers < 1) return fail("Direct J/K geometry workers must be positive");
  if ((order != 1 && order != 2) || (with_j != 0 && with_j != 1) || (with_k != 0 && with_k != 1) ||
      !(with_j || with_k))
    return fail("Invalid direct J/K geometry product");
  if (transpose && order != 2) return fail("order-1 VJP: use oracle_direct_jk_geometry_vjp");
  tables_t t;
  if (tables_init(&t, atm, natm, bas, nbas, env, nenv, cart)) { tables_free(&t); return 1; }
  if (n != t.n) { tables_free(&t); return fail("Direct J/K geometry density shape mismatch"); }
  const int nops = with_j + with_k;
  const size_t osize = transpose ? (size_t)nenv : (size_t)nops * nb * n * n;
  int w = workers < host_threads() ? workers : host_threads();
  if (w > t.nbas) w = t.nbas;
  double *partials = calloc((size_t)w * osize, sizeof(double));
  geo_task_t *tasks = calloc((size_t)w, sizeof(geo_task_t));
  pthread_t *threads = calloc((size_t)w, sizeof(pthread_t));
  for (int worker = 0; worker < w; ++worker) {
    geo_task_t task = {atm, natm, bas, nbas, env, nenv, cart, order, nb, with_j, with_k, transpose,
                       density, direction, vector, worker * t.nbas / w, (worker + 1) * t.nbas / w,
                       partials + (size_t)worker * osize};
    tasks[worker] = task;
  }
  for (int worker = 1; worker < w; ++worker) pthread_create(&threads[worker], NULL, geo_task_run, &tasks[worker]);
  geo_task_run(&tasks[0]);
  for (int worker = 1; worker < w; ++worker) pthread_join(threads[worker], NULL);
  free(tasks); free(threads);
  memset(out, 0, sizeof(double) * osize);
  for (int worker = 0; worker < w; ++worker)
    for (size_t i = 0; i < osize; ++i) out[i] += partials[(size_t)worker * osize + i];
  free(partials);
  tables_free(&t);
  return 0;
}

/* Unit of work: significant canonical contracted shell quartets
 * (i>=j, k>=l, ij>=kl, Q_ij*Q_kl >= cut), counted from the Schwarz table. */
long long oracle_count_quartets(const double *bounds, int nbas, double cut) {
  long long count = 0;
  const size_t npair = (size_t)nbas * (nbas + 1) / 2;
  double *q = malloc(sizeof(double) * npair);
  size_t m = 0;
  for (int i = 0; i < nbas; ++i)
    for (int j = 0; j <= i; ++j) q[m++] = bounds[(size_t)i * nbas + j];
  for (size_t a = 0; a < npair; ++a)
    for (size_t b = 0; b <= a; ++b)
      if (q[a] * q[b] >= cut) ++count;
  free(q);
  return count;
}
