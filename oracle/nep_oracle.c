/*
 * nep_oracle.c -- TEST INFRASTRUCTURE ONLY (see nep_oracle.h).
 *
 * Double-precision CPU restatement of the NEP4/NEP5/NEP-ZBL evaluation of
 * DMG-MD's single-rank path.  Every pair (center c, neighbour n, periodic
 * image) is an explicit directed edge; each edge adds its partial force
 * f = dE_c/dr_cn as F_c += f, F_n -= f and W_n += -r_cn (x) f.  That is the
 * attribution both reference kernel families use: the large-box gather
 * (src/gpumd_compat/nep.cu:756-881, src/gpumd_compat/potential.cu:81-210)
 * and the small-box scatter (src/gpumd_compat/nep_small_box.cuh:343-656).
 *
 * The angular partial force is the gradient of sum_{n,lm} a_{n,lm} g_n(d)
 * Y_lm(r/d) with a_{n,lm} = dE_c/ds_{n,lm}: the same quantity
 * accumulate_f12 (src/gpumd_compat/nep_utilities.cuh:1339-1491) evaluates
 * term by term.  The many-body invariants are held as monomial tables of the
 * polynomials written out in find_q (nep_utilities.cuh:1602-1730).
 */
#include "nep_oracle.h"

#include <ctype.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define MAXT 16
#define MAXN 17        /* basis_size + 1 */
#define LMAXH 8        /* largest l_max of the format */
#define NUM_ABC 80     /* (L_max+1)^2 - 1 for L_max = 8 */
#define MAX_DIM 256
#define MAX_INV 6
#define K_C_SP 14.399645
#define PI_D 3.14159265358979323846

/* element symbols, index = Z - 1 (reference nep.cu:37) */
static const char* kElements[94] = {
  "H", "He", "Li", "Be", "B", "C", "N", "O", "F", "Ne", "Na", "Mg", "Al", "Si", "P", "S",
  "Cl", "Ar", "K", "Ca", "Sc", "Ti", "V", "Cr", "Mn", "Fe", "Co", "Ni", "Cu", "Zn", "Ga", "Ge",
  "As", "Se", "Br", "Kr", "Rb", "Sr", "Y", "Zr", "Nb", "Mo", "Tc", "Ru", "Rh", "Pd", "Ag", "Cd",
  "In", "Sn", "Sb", "Te", "I", "Xe", "Cs", "Ba", "La", "Ce", "Pr", "Nd", "Pm", "Sm", "Eu", "Gd",
  "Tb", "Dy", "Ho", "Er", "Tm", "Yb", "Lu", "Hf", "Ta", "W", "Re", "Os", "Ir", "Pt", "Au", "Hg",
  "Tl", "Pb", "Bi", "Po", "At", "Rn", "Fr", "Ra", "Ac", "Th", "Pa", "U", "Np", "Pu"};

/* covalent radii used by the typewise ZBL cutoff (nep_utilities.cuh:175) */
static const double kCovalentRadius[94] = {
  0.426667, 0.613333, 1.6, 1.25333, 1.02667, 1.0, 0.946667, 0.84, 0.853333, 0.893333,
  1.86667, 1.66667, 1.50667, 1.38667, 1.46667, 1.36, 1.32, 1.28, 2.34667, 2.05333,
  1.77333, 1.62667, 1.61333, 1.46667, 1.42667, 1.38667, 1.33333, 1.32, 1.34667, 1.45333,
  1.49333, 1.45333, 1.53333, 1.46667, 1.52, 1.56, 2.52, 2.22667, 1.96, 1.85333,
  1.76, 1.65333, 1.53333, 1.50667, 1.50667, 1.44, 1.53333, 1.64, 1.70667, 1.68,
  1.68, 1.64, 1.76, 1.74667, 2.78667, 2.34667, 2.16, 1.96, 2.10667, 2.09333,
  2.08, 2.06667, 2.01333, 2.02667, 2.01333, 2.0, 1.98667, 1.98667, 1.97333, 2.04,
  1.94667, 1.82667, 1.74667, 1.64, 1.57333, 1.54667, 1.48, 1.49333, 1.50667, 1.76,
  1.73333, 1.73333, 1.81333, 1.74667, 1.84, 1.89333, 2.68, 2.41333, 2.22667, 2.10667,
  2.02667, 2.04, 2.05333, 2.06667};

/*
 * Real solid-harmonic building blocks.  For degree L and order m the
 * z-polynomial is sum_k kZ[L][m][k] z^k (z = cos theta); the full harmonic is
 * that polynomial times Re/Im (x + i y)^m.  kZ[L][m] is the primitive integer
 * polynomial (content divided out, positive leading coefficient) of
 * d^m P_L / dz^m, and kC3B the weight that makes
 *   q_L = kC3B[L0] s_L0^2 + 2 sum_{m>0} kC3B[Lm] (s_Lm,re^2 + s_Lm,im^2)
 * the rotation invariant sum_m |moment of the normalised Y_Lm|^2 (the
 * reference's Z_COEFFICIENT_L and C3B tables, nep_utilities.cuh:51-187).
 * Both come from Rodrigues' formula P_L = d^L/dz^L (z^2 - 1)^L / (2^L L!).
 */
static double kZ[LMAXH + 1][LMAXH + 1][LMAXH + 1];
static double kC3B[NUM_ABC];
static int g_harm_ready = 0;

static long long gcd_ll(long long a, long long b)
{
  if (a < 0) a = -a;
  if (b < 0) b = -b;
  while (b) {
    long long t = a % b;
    a = b;
    b = t;
  }
  return a;
}

static void build_harmonics(void)
{
  if (g_harm_ready) return;
  memset(kZ, 0, sizeof(kZ));
  for (int L = 1; L <= LMAXH; ++L) {
    /* (z^2 - 1)^L, coefficients of z^0 .. z^2L */
    long long w[2 * LMAXH + 1];
    memset(w, 0, sizeof(w));
    long long binom = 1;
    for (int k = 0; k <= L; ++k) {
      w[2 * k] = ((L - k) % 2 ? -1 : 1) * binom;
      binom = binom * (L - k) / (k + 1);
    }
    double lfact = 1.0;
    for (int r = 2; r <= L; ++r) lfact *= r;
    for (int m = 0; m <= L; ++m) {
      /* R = d^(L+m)/dz^(L+m) (z^2 - 1)^L, degree L - m */
      long long R[LMAXH + 1];
      long long g = 0;
      for (int k = 0; k <= L - m; ++k) {
        long long f = 1;
        for (int r = k + 1; r <= k + L + m; ++r) f *= r;
        R[k] = w[k + L + m] * f;
        g = gcd_ll(g, R[k]);
      }
      if (R[L - m] < 0) g = -g;
      for (int k = 0; k <= L - m; ++k) kZ[L][m][k] = (double)(R[k] / g);
      double kappa = (double)g / (ldexp(1.0, L) * lfact);
      double ratio = 1.0;
      for (int r = L - m + 1; r <= L + m; ++r) ratio /= r;
      double c = (2.0 * L + 1.0) / (4.0 * 3.14159265358979323846) * ratio * kappa * kappa;
      int st = L * L - 1;
      if (m == 0) {
        kC3B[st] = c;
      } else {
        kC3B[st + 2 * m - 1] = c;
        kC3B[st + 2 * m] = c;
      }
    }
  }
  g_harm_ready = 1;
}

void nepo_harmonic_tables(double* z, double* c3b)
{
  build_harmonics();
  if (z) memcpy(z, kZ, sizeof(kZ));
  if (c3b) memcpy(c3b, kC3B, sizeof(kC3B));
}

static const double kC4B[5] = {-0.007499480826664, -0.134990654879954, 0.067495327439977,
                               0.404971964639861, -0.809943929279723};
static const double kC5B[3] = {0.026596810706114, 0.053193621412227, 0.026596810706114};
static const double kC4B2[5] = {0.027493550848847, 0.164961305093080, -0.013746775424423,
                                0.041240326273270, 0.082480652546540};
static const double kC123[7] = {-0.008418146349617, -0.016836292699234, -0.033672585398469,
                                 -0.042090731748086, -0.067345170796937, -0.084181463496172,
                                 -0.168362926992344};
static const double kC233[10] = {0.008572620635186, 0.009644198214584, 0.019288396429168,
                                 0.025717861905558, 0.026789439484956, 0.032147327381947,
                                 0.038576792858337, 0.128589309527790, 0.192883964291685,
                                 0.321473273819474};
static const double kC134[10] = {0.003645164295772, 0.004860219061029, 0.006075273826286,
                                 0.018225821478859, 0.024301095305146, 0.036451642957719,
                                 0.042526916784005, 0.072903285915437, 0.085053833568010,
                                 0.255161500704030};

/* one monomial c * s[i0] s[i1] s[i2] (s[i3]); index -1 = absent */
typedef struct {
  double c;
  int i[4];
} mono_t;

#define MAX_MONO 40
typedef struct {
  int count;
  mono_t m[MAX_MONO];
} poly_t;

static void poly_add(poly_t* p, double c, int a, int b, int cc, int d)
{
  mono_t* t = &p->m[p->count++];
  t->c = c;
  t->i[0] = a;
  t->i[1] = b;
  t->i[2] = cc;
  t->i[3] = d;
}

/* many-body invariants as polynomials in the raw moments (find_q,
 * nep_utilities.cuh:1661-1728); order 222, 1111, 112, 123, 233, 134 */
static poly_t g_inv[MAX_INV];
static int g_inv_ready = 0;

static void build_invariants(void)
{
  if (g_inv_ready) return;
  memset(g_inv, 0, sizeof(g_inv));
  poly_t* p = &g_inv[0]; /* q_222 */
  poly_add(p, kC4B[0], 3, 3, 3, -1);
  poly_add(p, kC4B[1], 3, 4, 4, -1);
  poly_add(p, kC4B[1], 3, 5, 5, -1);
  poly_add(p, kC4B[2], 3, 6, 6, -1);
  poly_add(p, kC4B[2], 3, 7, 7, -1);
  poly_add(p, kC4B[3], 6, 5, 5, -1);
  poly_add(p, -kC4B[3], 6, 4, 4, -1);
  poly_add(p, kC4B[4], 4, 5, 7, -1);
  p = &g_inv[1]; /* q_1111 */
  poly_add(p, kC5B[0], 0, 0, 0, 0);
  poly_add(p, kC5B[1], 0, 0, 1, 1);
  poly_add(p, kC5B[1], 0, 0, 2, 2);
  poly_add(p, kC5B[2], 1, 1, 1, 1);
  poly_add(p, 2.0 * kC5B[2], 1, 1, 2, 2);
  poly_add(p, kC5B[2], 2, 2, 2, 2);
  p = &g_inv[2]; /* q_112 */
  poly_add(p, kC4B2[0], 0, 0, 3, -1);
  poly_add(p, kC4B2[1], 0, 1, 4, -1);
  poly_add(p, kC4B2[1], 0, 2, 5, -1);
  poly_add(p, kC4B2[2], 3, 1, 1, -1);
  poly_add(p, kC4B2[2], 3, 2, 2, -1);
  poly_add(p, kC4B2[3], 6, 1, 1, -1);
  poly_add(p, -kC4B2[3], 6, 2, 2, -1);
  poly_add(p, kC4B2[4], 1, 2, 7, -1);
  p = &g_inv[3]; /* q_123 */
  poly_add(p, kC123[6], 12, 2, 4, -1);
  poly_add(p, -kC123[6], 11, 2, 5, -1);
  poly_add(p, kC123[6], 1, 11, 4, -1);
  poly_add(p, kC123[6], 1, 12, 5, -1);
  poly_add(p, kC123[5], 0, 11, 6, -1);
  poly_add(p, kC123[5], 0, 12, 7, -1);
  poly_add(p, kC123[3], 14, 2, 6, -1);
  poly_add(p, -kC123[3], 13, 2, 7, -1);
  poly_add(p, kC123[3], 1, 13, 6, -1);
  poly_add(p, kC123[3], 1, 14, 7, -1);
  poly_add(p, kC123[4], 10, 0, 5, -1);
  poly_add(p, kC123[4], 0, 4, 9, -1);
  poly_add(p, kC123[1], 10, 2, 3, -1);
  poly_add(p, kC123[1], 0, 3, 8, -1);
  poly_add(p, kC123[1], 1, 3, 9, -1);
  poly_add(p, kC123[0], 10, 2, 6, -1);
  poly_add(p, -kC123[0], 10, 1, 7, -1);
  poly_add(p, -kC123[0], 2, 7, 9, -1);
  poly_add(p, -kC123[0], 1, 6, 9, -1);
  poly_add(p, -kC123[2], 2, 5, 8, -1);
  poly_add(p, -kC123[2], 1, 4, 8, -1);
  p = &g_inv[4]; /* q_233 */
  poly_add(p, kC233[0], 3, 8, 8, -1);
  poly_add(p, kC233[1], 10, 10, 3, -1);
  poly_add(p, kC233[1], 3, 9, 9, -1);
  poly_add(p, -kC233[2], 10, 10, 6, -1);
  poly_add(p, kC233[2], 6, 9, 9, -1);
  poly_add(p, kC233[3], 4, 8, 9, -1);
  poly_add(p, kC233[3], 10, 5, 8, -1);
  poly_add(p, -kC233[4], 13, 13, 3, -1);
  poly_add(p, -kC233[4], 14, 14, 3, -1);
  poly_add(p, -kC233[5], 14, 7, 9, -1);
  poly_add(p, -kC233[5], 13, 6, 9, -1);
  poly_add(p, -kC233[5], 10, 14, 6, -1);
  poly_add(p, kC233[5], 10, 13, 7, -1);
  poly_add(p, kC233[6], 10, 7, 9, -1);
  poly_add(p, -kC233[7], 11, 6, 8, -1);
  poly_add(p, -kC233[7], 12, 7, 8, -1);
  poly_add(p, kC233[8], 11, 4, 9, -1);
  poly_add(p, kC233[8], 12, 5, 9, -1);
  poly_add(p, kC233[8], 10, 12, 4, -1);
  poly_add(p, -kC233[8], 10, 11, 5, -1);
  poly_add(p, kC233[9], 12, 14, 4, -1);
  poly_add(p, kC233[9], 11, 14, 5, -1);
  poly_add(p, kC233[9], 13, 11, 4, -1);
  poly_add(p, -kC233[9], 13, 12, 5, -1);
  p = &g_inv[5]; /* q_134 */
  poly_add(p, -kC134[0], 10, 15, 2, -1);
  poly_add(p, -kC134[0], 1, 15, 9, -1);
  poly_add(p, kC134[1], 0, 15, 8, -1);
  poly_add(p, -kC134[2], 1, 13, 18, -1);
  poly_add(p, -kC134[2], 1, 14, 19, -1);
  poly_add(p, -kC134[2], 2, 14, 18, -1);
  poly_add(p, kC134[2], 2, 13, 19, -1);
  poly_add(p, -kC134[3], 10, 18, 2, -1);
  poly_add(p, kC134[3], 1, 10, 19, -1);
  poly_add(p, kC134[3], 1, 18, 9, -1);
  poly_add(p, kC134[3], 2, 19, 9, -1);
  poly_add(p, kC134[4], 1, 16, 8, -1);
  poly_add(p, kC134[4], 2, 17, 8, -1);
  poly_add(p, kC134[5], 0, 10, 17, -1);
  poly_add(p, kC134[5], 0, 16, 9, -1);
  poly_add(p, -kC134[5], 1, 11, 16, -1);
  poly_add(p, -kC134[5], 1, 12, 17, -1);
  poly_add(p, -kC134[5], 2, 12, 16, -1);
  poly_add(p, kC134[5], 2, 11, 17, -1);
  poly_add(p, kC134[6], 1, 13, 22, -1);
  poly_add(p, kC134[6], 1, 14, 23, -1);
  poly_add(p, -kC134[6], 2, 14, 22, -1);
  poly_add(p, kC134[6], 2, 13, 23, -1);
  poly_add(p, kC134[7], 0, 11, 18, -1);
  poly_add(p, kC134[7], 0, 12, 19, -1);
  poly_add(p, kC134[8], 0, 13, 20, -1);
  poly_add(p, kC134[8], 0, 14, 21, -1);
  poly_add(p, kC134[9], 1, 11, 20, -1);
  poly_add(p, kC134[9], 1, 12, 21, -1);
  poly_add(p, -kC134[9], 2, 12, 20, -1);
  poly_add(p, kC134[9], 2, 11, 21, -1);
  g_inv_ready = 1;
}

static double poly_eval(const poly_t* p, const double* s)
{
  double q = 0.0;
  for (int k = 0; k < p->count; ++k) {
    const mono_t* t = &p->m[k];
    double v = t->c;
    for (int f = 0; f < 4 && t->i[f] >= 0; ++f) v *= s[t->i[f]];
    q += v;
  }
  return q;
}

/* grad[j] += w * d poly / d s[j] */
static void poly_grad(const poly_t* p, const double* s, double w, double* grad)
{
  for (int k = 0; k < p->count; ++k) {
    const mono_t* t = &p->m[k];
    int nf = 0;
    while (nf < 4 && t->i[nf] >= 0) ++nf;
    for (int f = 0; f < nf; ++f) {
      double v = w * t->c;
      for (int g = 0; g < nf; ++g)
        if (g != f) v *= s[t->i[g]];
      grad[t->i[f]] += v;
    }
  }
}

struct nepo_model {
  int version;
  int zbl, zbl_flexible, typewise_zbl;
  double typewise_factor, rc_inner, rc_outer;
  double zbl_para[550];
  int num_types;
  int Z[MAXT];
  double rc_r[MAXT], rc_a[MAXT], rc_r_max;
  int MN_r, MN_a;
  int nmax_r, nmax_a, basis_r, basis_a, L_max;
  int has_inv[MAX_INV];
  int num_L, dim_angular, dim, H;
  int num_para_ann, num_c_radial;
  double* params; /* file order: ANN block, descriptor block, q_scaler */
  double* c_pair; /* type-pair major radial block then angular block */
  const double *w0[MAXT], *b0[MAXT], *w1[MAXT];
  const double* b1;
  const double* q_scaler;
};

/* ---------------------------------------------------------------- parsing */

typedef struct {
  FILE* f;
  char line[4096];
  char* tok[64];
  int ntok;
} reader_t;

static int next_line(reader_t* r)
{
  while (fgets(r->line, sizeof(r->line), r->f)) {
    r->ntok = 0;
    char* p = r->line;
    while (*p && r->ntok < 64) {
      while (*p && isspace((unsigned char)*p)) ++p;
      if (!*p) break;
      r->tok[r->ntok++] = p;
      while (*p && !isspace((unsigned char)*p)) ++p;
      if (*p) *p++ = '\0';
    }
    if (r->ntok > 0) return 1;
  }
  r->ntok = 0;
  return 0;
}

#define FAIL(...)                                  \
  do {                                             \
    if (err) snprintf(err, errlen, __VA_ARGS__);   \
    goto fail;                                     \
  } while (0)

nepo_model* nepo_load(const char* path, char* err, int errlen)
{
  build_invariants();
  build_harmonics();
  reader_t r;
  memset(&r, 0, sizeof(r));
  nepo_model* m = (nepo_model*)calloc(1, sizeof(nepo_model));
  r.f = fopen(path, "r");
  if (!r.f) FAIL("cannot open %s", path);
  if (!next_line(&r) || r.ntok < 3) FAIL("first line needs at least 3 items");
  if (!strcmp(r.tok[0], "nep4")) {
    m->version = 4;
  } else if (!strcmp(r.tok[0], "nep4_zbl")) {
    m->version = 4;
    m->zbl = 1;
  } else if (!strcmp(r.tok[0], "nep5")) {
    m->version = 5;
  } else if (!strcmp(r.tok[0], "nep5_zbl")) {
    m->version = 5;
    m->zbl = 1;
  } else {
    FAIL("unsupported model %s", r.tok[0]);
  }
  m->num_types = atoi(r.tok[1]);
  if (m->num_types < 1 || m->num_types > MAXT) FAIL("bad number of types");
  if (r.ntok != 2 + m->num_types) FAIL("first line needs %d symbols", m->num_types);
  for (int t = 0; t < m->num_types; ++t) {
    m->Z[t] = 0;
    for (int e = 0; e < 94; ++e)
      if (!strcmp(r.tok[2 + t], kElements[e])) m->Z[t] = e + 1;
  }
  if (m->zbl) {
    if (!next_line(&r) || (r.ntok != 3 && r.ntok != 4)) FAIL("zbl line");
    m->rc_inner = atof(r.tok[1]);
    m->rc_outer = atof(r.tok[2]);
    if (m->rc_inner == 0 && m->rc_outer == 0) {
      m->zbl_flexible = 1;
    } else if (r.ntok == 4) {
      m->typewise_zbl = 1;
      m->typewise_factor = atof(r.tok[3]);
    }
  }
  if (!next_line(&r)) FAIL("missing cutoff line");
  if (r.ntok == 5) {
    for (int t = 0; t < m->num_types; ++t) {
      m->rc_r[t] = atof(r.tok[1]);
      m->rc_a[t] = atof(r.tok[2]);
    }
  } else if (r.ntok == 2 * m->num_types + 3) {
    for (int t = 0; t < m->num_types; ++t) {
      m->rc_r[t] = atof(r.tok[1 + 2 * t]);
      m->rc_a[t] = atof(r.tok[2 + 2 * t]);
    }
  } else {
    FAIL("cutoff line has %d items", r.ntok);
  }
  for (int t = 0; t < m->num_types; ++t)
    if (m->rc_r[t] > m->rc_r_max) m->rc_r_max = m->rc_r[t];
  m->MN_r = (int)ceil(atoi(r.tok[r.ntok - 2]) * 1.25);
  m->MN_a = (int)ceil(atoi(r.tok[r.ntok - 1]) * 1.25);
  if (!next_line(&r) || r.ntok != 3) FAIL("n_max line");
  m->nmax_r = atoi(r.tok[1]);
  m->nmax_a = atoi(r.tok[2]);
  if (!next_line(&r) || r.ntok != 3) FAIL("basis_size line");
  m->basis_r = atoi(r.tok[1]);
  m->basis_a = atoi(r.tok[2]);
  if (m->basis_r + 1 > MAXN || m->basis_a + 1 > MAXN) FAIL("basis too large");
  if (!next_line(&r) || r.ntok < 4) FAIL("l_max line");
  m->L_max = atoi(r.tok[1]);
  if (m->L_max < 0 || m->L_max > LMAXH) FAIL("oracle supports l_max <= 8");
  m->num_L = m->L_max;
  for (int k = 0; k < MAX_INV; ++k) {
    m->has_inv[k] = (2 + k < r.ntok) ? atoi(r.tok[2 + k]) : 0;
    if (m->has_inv[k]) m->num_L += 1;
  }
  m->dim_angular = (m->nmax_a + 1) * m->num_L;
  if (!next_line(&r) || r.ntok != 3) FAIL("ANN line");
  m->H = atoi(r.tok[1]);
  m->dim = (m->nmax_r + 1) + m->dim_angular;
  if (m->dim > MAX_DIM) FAIL("descriptor too long");
  int T = m->num_types;
  if (m->version == 4)
    m->num_para_ann = (m->dim + 2) * m->H * T + 1;
  else
    m->num_para_ann = ((m->dim + 2) * m->H + 1) * T + 1;
  int kR = m->basis_r + 1, kA = m->basis_a + 1;
  int nR = m->nmax_r + 1, nA = m->nmax_a + 1;
  m->num_c_radial = T * T * nR * kR;
  int num_desc = T * T * (nR * kR + nA * kA);
  int total = m->num_para_ann + num_desc + m->dim;
  m->params = (double*)malloc(sizeof(double) * total);
  for (int k = 0; k < total; ++k) {
    if (!next_line(&r)) FAIL("file ends after %d of %d parameters", k, total);
    m->params[k] = atof(r.tok[0]);
  }
  if (m->zbl_flexible) {
    int npair = T * (T + 1) / 2;
    for (int k = 0; k < 10 * npair; ++k) {
      if (!next_line(&r)) FAIL("missing flexible ZBL parameter");
      m->zbl_para[k] = atof(r.tok[0]);
    }
  }
  /* ANN views (nep.cu:464-496) */
  const double* p = m->params;
  for (int t = 0; t < T; ++t) {
    m->w0[t] = p;
    p += m->H * m->dim;
    m->b0[t] = p;
    p += m->H;
    m->w1[t] = p;
    p += m->H;
    if (m->version == 5) p += 1;
  }
  m->b1 = p;
  /* descriptor coefficients: file is basis-major, kernels want pair-major
     (nep.cu:103-126) */
  m->c_pair = (double*)malloc(sizeof(double) * num_desc);
  for (int tp = 0; tp < T * T; ++tp) {
    for (int b = 0; b < nR * kR; ++b)
      m->c_pair[tp * nR * kR + b] = m->params[m->num_para_ann + b * T * T + tp];
    for (int b = 0; b < nA * kA; ++b)
      m->c_pair[m->num_c_radial + tp * nA * kA + b] =
        m->params[m->num_para_ann + m->num_c_radial + b * T * T + tp];
  }
  m->q_scaler = m->params + m->num_para_ann + num_desc;
  fclose(r.f);
  return m;
fail:
  if (r.f) fclose(r.f);
  nepo_free(m);
  return NULL;
}

void nepo_free(nepo_model* m)
{
  if (!m) return;
  free(m->params);
  free(m->c_pair);
  free(m);
}

void nepo_info(const nepo_model* m, int* info, double* rc)
{
  int mask = 0;
  for (int k = 0; k < MAX_INV; ++k)
    if (m->has_inv[k]) mask |= 1 << k;
  int v[16] = {m->version, m->num_types, m->zbl,  m->zbl_flexible, m->nmax_r, m->nmax_a,
               m->basis_r, m->basis_a,   m->L_max, m->num_L,        m->dim,    m->H,
               m->MN_r,    m->MN_a,      mask,     m->typewise_zbl};
  memcpy(info, v, sizeof(v));
  if (rc) {
    for (int t = 0; t < m->num_types; ++t) {
      rc[2 * t] = m->rc_r[t];
      rc[2 * t + 1] = m->rc_a[t];
    }
  }
}

/* ---------------------------------------------------------------- geometry */

typedef struct {
  double h[9], hinv[9];
  int pbc[3];
  int img[3]; /* images per direction searched on each side */
} box_t;

static void box_setup(box_t* b, const double* h, const int* pbc, double rc)
{
  memcpy(b->h, h, sizeof(double) * 9);
  memcpy(b->pbc, pbc, sizeof(int) * 3);
  const double* a = h;
  double det = a[0] * (a[4] * a[8] - a[5] * a[7]) + a[1] * (a[5] * a[6] - a[3] * a[8]) +
               a[2] * (a[3] * a[7] - a[4] * a[6]);
  b->hinv[0] = (a[4] * a[8] - a[5] * a[7]) / det;
  b->hinv[1] = (a[2] * a[7] - a[1] * a[8]) / det;
  b->hinv[2] = (a[1] * a[5] - a[2] * a[4]) / det;
  b->hinv[3] = (a[5] * a[6] - a[3] * a[8]) / det;
  b->hinv[4] = (a[0] * a[8] - a[2] * a[6]) / det;
  b->hinv[5] = (a[2] * a[3] - a[0] * a[5]) / det;
  b->hinv[6] = (a[3] * a[7] - a[4] * a[6]) / det;
  b->hinv[7] = (a[1] * a[6] - a[0] * a[7]) / det;
  b->hinv[8] = (a[0] * a[4] - a[1] * a[3]) / det;
  double vol = fabs(det);
  /* thickness along each cell vector = volume / area of the opposite face */
  for (int d = 0; d < 3; ++d) {
    int e = (d + 1) % 3, f = (d + 2) % 3;
    double u[3] = {h[e], h[3 + e], h[6 + e]}, w[3] = {h[f], h[3 + f], h[6 + f]};
    double cx = u[1] * w[2] - u[2] * w[1], cy = u[2] * w[0] - u[0] * w[2],
           cz = u[0] * w[1] - u[1] * w[0];
    double thick = vol / sqrt(cx * cx + cy * cy + cz * cz);
    /* |r| < rc implies |s_d| < rc / thick_d, so a box thicker than 2 rc needs
       only the fractional minimum image */
    b->img[d] = (pbc[d] && thick <= 2.0 * rc) ? (int)ceil(rc / thick + 0.5) : 0;
  }
}

/* fractional minimum image of a double displacement */
static void mic(const box_t* b, double* r)
{
  double s[3];
  for (int d = 0; d < 3; ++d)
    s[d] = b->hinv[3 * d] * r[0] + b->hinv[3 * d + 1] * r[1] + b->hinv[3 * d + 2] * r[2];
  for (int d = 0; d < 3; ++d)
    if (b->pbc[d]) s[d] -= nearbyint(s[d]);
  for (int d = 0; d < 3; ++d) r[d] = b->h[3 * d] * s[0] + b->h[3 * d + 1] * s[1] + b->h[3 * d + 2] * s[2];
}

typedef struct {
  int c, n;     /* center, neighbour */
  double r[3];  /* r_n - r_c including the periodic image */
  double d;
} edge_t;

typedef struct {
  edge_t* e;
  int count, cap;
  int* start; /* per center, edges sorted by center */
} edges_t;

static void edges_push(edges_t* E, int c, int n, const double* r, double d)
{
  if (E->count == E->cap) {
    E->cap = E->cap ? 2 * E->cap : 1024;
    E->e = (edge_t*)realloc(E->e, sizeof(edge_t) * E->cap);
  }
  edge_t* x = &E->e[E->count++];
  x->c = c;
  x->n = n;
  x->r[0] = r[0];
  x->r[1] = r[1];
  x->r[2] = r[2];
  x->d = d;
}

/*
 * All directed edges with |r| < rc_max (the largest type-pair cutoff), every
 * periodic image included.  Equivalent to the large-box minimum image when
 * the box is thicker than twice the cutoff, and to the explicit image
 * enumeration of the small-box path (nep_small_box.cuh:96-176) otherwise.
 */
static void build_edges(const box_t* b, int n, const double* pos, double rc_max, edges_t* E)
{
  E->count = 0;
  E->start = (int*)calloc(n + 1, sizeof(int));
  const double* x = pos;
  const double* y = pos + n;
  const double* z = pos + 2 * n;
  double rc2 = rc_max * rc_max;
  for (int i = 0; i < n; ++i) {
    E->start[i] = E->count;
    for (int j = 0; j < n; ++j) {
      double r0[3] = {x[j] - x[i], y[j] - y[i], z[j] - z[i]};
      mic(b, r0);
      for (int ia = -b->img[0]; ia <= b->img[0]; ++ia)
        for (int ib = -b->img[1]; ib <= b->img[1]; ++ib)
          for (int ic = -b->img[2]; ic <= b->img[2]; ++ic) {
            if (i == j && ia == 0 && ib == 0 && ic == 0) continue;
            double r[3];
            for (int d = 0; d < 3; ++d)
              r[d] = r0[d] + b->h[3 * d] * ia + b->h[3 * d + 1] * ib + b->h[3 * d + 2] * ic;
            double d2 = r[0] * r[0] + r[1] * r[1] + r[2] * r[2];
            if (d2 < rc2) edges_push(E, i, j, r, sqrt(d2));
          }
    }
  }
  E->start[n] = E->count;
}

/* ---------------------------------------------------------------- basis */

/* cutoff function and derivative (nep_utilities.cuh:317-345) */
static void fc_fcp(double rc, double d, double* fc, double* fcp)
{
  if (d < rc) {
    double x = d / rc;
    *fc = 0.5 * cos(PI_D * x) + 0.5;
    *fcp = -0.5 * PI_D / rc * sin(PI_D * x);
  } else {
    *fc = 0.0;
    *fcp = 0.0;
  }
}

/* shifted Chebyshev basis times fc and its d-derivative (nep_utilities.cuh:440-497) */
static void basis(int kmax, double rc, double d, double* fn, double* fnp)
{
  double fc, fcp;
  fc_fcp(rc, d, &fc, &fcp);
  double u = d / rc - 1.0;
  double x = 2.0 * u * u - 1.0;
  double dx = 4.0 * u / rc;
  double T0 = 1.0, T1 = x, dT0 = 0.0, dT1 = 1.0;
  fn[0] = fc;
  fnp[0] = fcp;
  if (kmax >= 1) {
    fn[1] = 0.5 * (x + 1.0) * fc;
    fnp[1] = 0.5 * dx * fc + 0.5 * (x + 1.0) * fcp;
  }
  for (int k = 2; k <= kmax; ++k) {
    double T2 = 2.0 * x * T1 - T0;
    double dT2 = 2.0 * T1 + 2.0 * x * dT1 - dT0;
    fn[k] = 0.5 * (T2 + 1.0) * fc;
    fnp[k] = 0.5 * dT2 * dx * fc + 0.5 * (T2 + 1.0) * fcp;
    T0 = T1;
    T1 = T2;
    dT0 = dT1;
    dT1 = dT2;
  }
}

/*
 * Y[lm] and grad[lm][3] of the unnormalised real harmonics at unit vector u,
 * gradient taken with respect to the un-normalised displacement r (|r| = d):
 * the ladder of accumulate_s_one / accumulate_f12_one
 * (nep_utilities.cuh:1240-1335, 1547-1581).
 */
static void harmonics(int L_max, const double* u, double d, double* Y, double (*G)[3])
{
  double dinv = 1.0 / d;
  double dxv[3] = {(1.0 - u[0] * u[0]) * dinv, -u[0] * u[1] * dinv, -u[0] * u[2] * dinv};
  double dyv[3] = {-u[0] * u[1] * dinv, (1.0 - u[1] * u[1]) * dinv, -u[1] * u[2] * dinv};
  double dzv[3] = {-u[0] * u[2] * dinv, -u[1] * u[2] * dinv, (1.0 - u[2] * u[2]) * dinv};
  int idx = 0;
  for (int L = 1; L <= L_max; ++L) {
    double zp[LMAXH + 1];
    zp[0] = 1.0;
    for (int k = 1; k <= L; ++k) zp[k] = zp[k - 1] * u[2];
    double re = 1.0, im = 0.0; /* (x + i y)^(m-1) */
    for (int m = 0; m <= L; ++m) {
      double zf = 0.0, dzf = 0.0;
      for (int k = (L + m) % 2; k <= L - m; k += 2) {
        zf += kZ[L][m][k] * zp[k];
        if (k > 0) dzf += kZ[L][m][k] * k * zp[k - 1];
      }
      if (m == 0) {
        Y[idx] = zf;
        for (int c = 0; c < 3; ++c) G[idx][c] = dzf * dzv[c];
        ++idx;
      } else {
        /* d/dr of Re,Im (x+iy)^m = m (x+iy)^(m-1) (dx + i dy) */
        double pre = re * u[0] - im * u[1], pim = re * u[1] + im * u[0]; /* (x+iy)^m */
        for (int c = 0; c < 3; ++c) {
          double dre = m * (re * dxv[c] - im * dyv[c]);
          double dim = m * (re * dyv[c] + im * dxv[c]);
          G[idx][c] = dre * zf + pre * dzf * dzv[c];
          G[idx + 1][c] = dim * zf + pim * dzf * dzv[c];
        }
        Y[idx] = pre * zf;
        Y[idx + 1] = pim * zf;
        idx += 2;
        re = pre;
        im = pim;
      }
    }
  }
}

/* ---------------------------------------------------------------- evaluation */

typedef struct {
  double q[MAX_DIM];        /* scaled descriptor */
  double Fp[MAX_DIM];       /* dE/dq_unscaled, i.e. dE/dq * q_scaler */
  double a[MAXN * NUM_ABC]; /* dE/ds[n][lm] */
  double s[MAXN * NUM_ABC];
  double e;
} center_t;

static double pair_rc(const double* rc, int t1, int t2) { return 0.5 * (rc[t1] + rc[t2]); }

static void descriptor_and_ann(const nepo_model* m, const edges_t* E, const int* type, int i,
                               center_t* C, int want_ann)
{
  int T = m->num_types, nR = m->nmax_r + 1, nA = m->nmax_a + 1;
  int kR = m->basis_r + 1, kA = m->basis_a + 1;
  int nabc = (m->L_max + 1) * (m->L_max + 1) - 1;
  int t1 = type[i];
  double q[MAX_DIM];
  memset(q, 0, sizeof(q));
  memset(C->s, 0, sizeof(C->s));
  for (int k = E->start[i]; k < E->start[i + 1]; ++k) {
    const edge_t* e = &E->e[k];
    int t2 = type[e->n];
    double fn[MAXN], fnp[MAXN];
    double rcr = pair_rc(m->rc_r, t1, t2);
    if (e->d < rcr) {
      basis(m->basis_r, rcr, e->d, fn, fnp);
      const double* c = m->c_pair + (t1 * T + t2) * nR * kR;
      for (int n = 0; n < nR; ++n) {
        double g = 0.0;
        for (int b = 0; b < kR; ++b) g += fn[b] * c[n * kR + b];
        q[n] += g;
      }
    }
    double rca = pair_rc(m->rc_a, t1, t2);
    if (e->d < rca) {
      basis(m->basis_a, rca, e->d, fn, fnp);
      const double* c = m->c_pair + m->num_c_radial + (t1 * T + t2) * nA * kA;
      double u[3] = {e->r[0] / e->d, e->r[1] / e->d, e->r[2] / e->d};
      double Y[NUM_ABC], G[NUM_ABC][3];
      harmonics(m->L_max, u, e->d, Y, G);
      for (int n = 0; n < nA; ++n) {
        double g = 0.0;
        for (int b = 0; b < kA; ++b) g += fn[b] * c[n * kA + b];
        for (int lm = 0; lm < nabc; ++lm) C->s[n * NUM_ABC + lm] += g * Y[lm];
      }
    }
  }
  /* invariants (find_q) */
  for (int n = 0; n < nA; ++n) {
    const double* s = C->s + n * NUM_ABC;
    int col = 0;
    for (int L = 1; L <= m->L_max; ++L, ++col) {
      int st = L * L - 1;
      double v = 0.0;
      for (int k = 1; k < 2 * L + 1; ++k) v += kC3B[st + k] * s[st + k] * s[st + k];
      v = 2.0 * v + kC3B[st] * s[st] * s[st];
      q[nR + col * nA + n] = v;
    }
    for (int inv = 0; inv < MAX_INV; ++inv)
      if (m->has_inv[inv]) q[nR + (col++) * nA + n] = poly_eval(&g_inv[inv], s);
  }
  for (int d = 0; d < m->dim; ++d) C->q[d] = q[d] * m->q_scaler[d];
  if (!want_ann) return;
  /* one hidden layer tanh ANN (nep_utilities.cuh:169-315) */
  double Ei = 0.0, dE[MAX_DIM];
  memset(dE, 0, sizeof(dE));
  const double* w0 = m->w0[t1];
  for (int h = 0; h < m->H; ++h) {
    double z = 0.0;
    for (int d = 0; d < m->dim; ++d) z += w0[h * m->dim + d] * C->q[d];
    double x1 = tanh(z - m->b0[t1][h]);
    double dx = 1.0 - x1 * x1;
    Ei += m->w1[t1][h] * x1;
    for (int d = 0; d < m->dim; ++d) dE[d] += m->w1[t1][h] * dx * w0[h * m->dim + d];
  }
  if (m->version == 5)
    Ei -= m->w1[t1][m->H] + m->b1[0];
  else
    Ei -= m->b1[0];
  C->e = Ei;
  for (int d = 0; d < m->dim; ++d) C->Fp[d] = dE[d] * m->q_scaler[d];
  /* a[n][lm] = dE/ds[n][lm] */
  memset(C->a, 0, sizeof(C->a));
  for (int n = 0; n < nA; ++n) {
    const double* s = C->s + n * NUM_ABC;
    double* a = C->a + n * NUM_ABC;
    int col = 0;
    for (int L = 1; L <= m->L_max; ++L, ++col) {
      double fp = C->Fp[nR + col * nA + n];
      int st = L * L - 1;
      a[st] += 2.0 * fp * kC3B[st] * s[st];
      for (int k = 1; k < 2 * L + 1; ++k) a[st + k] += 4.0 * fp * kC3B[st + k] * s[st + k];
    }
    for (int inv = 0; inv < MAX_INV; ++inv)
      if (m->has_inv[inv]) poly_grad(&g_inv[inv], s, C->Fp[nR + (col++) * nA + n], a);
  }
}

/* universal / flexible ZBL energy and d/dd (nep_utilities.cuh:378-475) */
static void zbl_pair(const nepo_model* m, int t1, int t2, double d, double* f, double* fp)
{
  int zi = m->Z[t1], zj = m->Z[t2];
  double a_inv = (pow((double)zi, 0.23) + pow((double)zj, 0.23)) * 2.134563;
  double zizj = K_C_SP * zi * zj;
  double x = d * a_inv, dinv = 1.0 / d;
  double phi = 0.0, phip = 0.0, r1, r2;
  if (m->zbl_flexible) {
    int a = t1 < t2 ? t1 : t2, b = t1 < t2 ? t2 : t1;
    int idx = a * m->num_types - (a * (a - 1)) / 2 + (b - a);
    const double* p = m->zbl_para + 10 * idx;
    for (int k = 0; k < 4; ++k) {
      double t = p[2 + 2 * k] * exp(-p[3 + 2 * k] * x);
      phi += t;
      phip -= p[3 + 2 * k] * t;
    }
    r1 = p[0];
    r2 = p[1];
  } else {
    static const double kp[8] = {0.18175, 3.1998, 0.50986, 0.94229,
                                 0.28022, 0.4029, 0.02817, 0.20162};
    for (int k = 0; k < 4; ++k) {
      double t = kp[2 * k] * exp(-kp[2 * k + 1] * x);
      phi += t;
      phip -= kp[2 * k + 1] * t;
    }
    r1 = m->rc_inner;
    r2 = m->rc_outer;
    if (m->typewise_zbl) {
      double rt = (kCovalentRadius[zi - 1] + kCovalentRadius[zj - 1]) * m->typewise_factor;
      r2 = rt < r2 ? rt : r2;
      r1 = 0.0;
    }
  }
  double ff = phi * zizj;
  double ffp = phip * zizj * a_inv;
  ffp = ffp * dinv - ff * dinv * dinv;
  ff *= dinv;
  double fc, fcp;
  if (d < r1) {
    fc = 1.0;
    fcp = 0.0;
  } else if (d < r2) {
    double pf = PI_D / (r2 - r1);
    fc = 0.5 * cos(pf * (d - r1)) + 0.5;
    fcp = -0.5 * sin(pf * (d - r1)) * pf;
  } else {
    fc = 0.0;
    fcp = 0.0;
  }
  *fp = ffp * fc + ff * fcp;
  *f = ff * fc;
}

static void add_edge(int c, int nb, const double* r, const double* f, int n, double* force,
                     double* virial)
{
  force[c] += f[0];
  force[n + c] += f[1];
  force[2 * n + c] += f[2];
  force[nb] -= f[0];
  force[n + nb] -= f[1];
  force[2 * n + nb] -= f[2];
  /* W_nb += -r (x) f in the order xx yy zz xy xz yz yx zx zy */
  virial[0 * n + nb] -= r[0] * f[0];
  virial[1 * n + nb] -= r[1] * f[1];
  virial[2 * n + nb] -= r[2] * f[2];
  virial[3 * n + nb] -= r[0] * f[1];
  virial[4 * n + nb] -= r[0] * f[2];
  virial[5 * n + nb] -= r[1] * f[2];
  virial[6 * n + nb] -= r[1] * f[0];
  virial[7 * n + nb] -= r[2] * f[0];
  virial[8 * n + nb] -= r[2] * f[1];
}

static double max_cutoff(const nepo_model* m)
{
  double rc = 0.0;
  for (int t = 0; t < m->num_types; ++t) {
    if (m->rc_r[t] > rc) rc = m->rc_r[t];
    if (m->rc_a[t] > rc) rc = m->rc_a[t];
  }
  return rc;
}

int nepo_compute(const nepo_model* m, int n, const int* type, const double* h, const int* pbc,
                 const double* pos, double* pe, double* force, double* virial)
{
  box_t b;
  double rc = max_cutoff(m);
  box_setup(&b, h, pbc, rc);
  edges_t E;
  memset(&E, 0, sizeof(E));
  build_edges(&b, n, pos, rc, &E);
  center_t* C = (center_t*)malloc(sizeof(center_t) * (n > 0 ? n : 1));
  for (int i = 0; i < n; ++i) descriptor_and_ann(m, &E, type, i, &C[i], 1);
  memset(force, 0, sizeof(double) * 3 * n);
  memset(virial, 0, sizeof(double) * 9 * n);
  int T = m->num_types, nR = m->nmax_r + 1, nA = m->nmax_a + 1;
  int kR = m->basis_r + 1, kA = m->basis_a + 1;
  int nabc = (m->L_max + 1) * (m->L_max + 1) - 1;
  for (int i = 0; i < n; ++i) pe[i] = C[i].e;
  for (int k = 0; k < E.count; ++k) {
    const edge_t* e = &E.e[k];
    int i = e->c, t1 = type[i], t2 = type[e->n];
    double u[3] = {e->r[0] / e->d, e->r[1] / e->d, e->r[2] / e->d};
    double f[3] = {0.0, 0.0, 0.0};
    double fn[MAXN], fnp[MAXN];
    /* radial: dE_i/dr_ij = sum_n Fp_i[n] g'_n(d) u */
    double rcr = pair_rc(m->rc_r, t1, t2);
    if (e->d < rcr) {
      basis(m->basis_r, rcr, e->d, fn, fnp);
      const double* c = m->c_pair + (t1 * T + t2) * nR * kR;
      double w = 0.0;
      for (int nn = 0; nn < nR; ++nn) {
        double gp = 0.0;
        for (int bb = 0; bb < kR; ++bb) gp += fnp[bb] * c[nn * kR + bb];
        w += C[i].Fp[nn] * gp;
      }
      for (int d = 0; d < 3; ++d) f[d] += w * u[d];
    }
    /* angular: gradient of sum a[n][lm] g_n Y_lm */
    double rca = pair_rc(m->rc_a, t1, t2);
    if (e->d < rca) {
      basis(m->basis_a, rca, e->d, fn, fnp);
      const double* c = m->c_pair + m->num_c_radial + (t1 * T + t2) * nA * kA;
      double Y[NUM_ABC], G[NUM_ABC][3];
      harmonics(m->L_max, u, e->d, Y, G);
      for (int nn = 0; nn < nA; ++nn) {
        double g = 0.0, gp = 0.0;
        for (int bb = 0; bb < kA; ++bb) {
          g += fn[bb] * c[nn * kA + bb];
          gp += fnp[bb] * c[nn * kA + bb];
        }
        const double* a = C[i].a + nn * NUM_ABC;
        for (int lm = 0; lm < nabc; ++lm) {
          double al = a[lm];
          for (int d = 0; d < 3; ++d) f[d] += al * (gp * Y[lm] * u[d] + g * G[lm][d]);
        }
      }
      if (m->zbl) {
        double zf, zfp;
        zbl_pair(m, t1, t2, e->d, &zf, &zfp);
        pe[i] += 0.5 * zf;
        for (int d = 0; d < 3; ++d) f[d] += 0.5 * zfp * u[d];
      }
    }
    add_edge(i, e->n, e->r, f, n, force, virial);
  }
  free(C);
  free(E.e);
  free(E.start);
  return 0;
}

int nepo_descriptors(const nepo_model* m, int n, const int* type, const double* h,
                     const int* pbc, const double* pos, double* q)
{
  box_t b;
  double rc = max_cutoff(m);
  box_setup(&b, h, pbc, rc);
  edges_t E;
  memset(&E, 0, sizeof(E));
  build_edges(&b, n, pos, rc, &E);
  center_t C;
  for (int i = 0; i < n; ++i) {
    descriptor_and_ann(m, &E, type, i, &C, 0);
    memcpy(q + (size_t)i * m->dim, C.q, sizeof(double) * m->dim);
  }
  free(E.e);
  free(E.start);
  return 0;
}

/* float minimum image of the large-box path (box.cuh:84-127) */
static void mic_f32(const float* fh, int ortho, const int* pbc, float* x, float* y, float* z)
{
  if (ortho) {
    float L[3] = {fh[0], fh[4], fh[8]};
    float* v[3] = {x, y, z};
    for (int d = 0; d < 3; ++d) {
      if (!pbc[d]) continue;
      float half = L[d] * 0.5f;
      if (*v[d] < -half)
        *v[d] += L[d];
      else if (*v[d] > +half)
        *v[d] -= L[d];
    }
  } else {
    float sx = fh[9] * *x + fh[10] * *y + fh[11] * *z;
    float sy = fh[12] * *x + fh[13] * *y + fh[14] * *z;
    float sz = fh[15] * *x + fh[16] * *y + fh[17] * *z;
    if (pbc[0]) sx -= nearbyintf(sx);
    if (pbc[1]) sy -= nearbyintf(sy);
    if (pbc[2]) sz -= nearbyintf(sz);
    *x = fh[0] * sx + fh[1] * sy + fh[2] * sz;
    *y = fh[3] * sx + fh[4] * sy + fh[5] * sz;
    *z = fh[6] * sx + fh[7] * sy + fh[8] * sz;
  }
}

int nepo_neighbors_f32(const nepo_model* m, int n, const int* type, const double* h,
                       const int* pbc, const double* pos, int which, int mn, int* nn, int* nl)
{
  box_t b;
  box_setup(&b, h, pbc, 1.0);
  float fh[18];
  for (int k = 0; k < 9; ++k) {
    fh[k] = (float)h[k];
    fh[9 + k] = (float)b.hinv[k];
  }
  int ortho = h[1] == 0 && h[2] == 0 && h[3] == 0 && h[5] == 0 && h[6] == 0 && h[7] == 0;
  const double* x = pos;
  const double* y = pos + n;
  const double* z = pos + 2 * n;
  int overflow = 0;
  for (int i = 0; i < n; ++i) {
    int cnt = 0;
    for (int j = 0; j < n; ++j) {
      if (j == i) continue;
      float dx = (float)(x[j] - x[i]);
      float dy = (float)(y[j] - y[i]);
      float dz = (float)(z[j] - z[i]);
      mic_f32(fh, ortho, pbc, &dx, &dy, &dz);
      /* the reference's d2 expression as nvcc contracts it into two FMAs */
      float d2 = fmaf(dz, dz, fmaf(dx, dx, dy * dy));
      const double* rcv = which == 0 ? m->rc_r : m->rc_a;
      float rcf = ((float)rcv[type[i]] + (float)rcv[type[j]]) * 0.5f;
      if (d2 < rcf * rcf) {
        if (cnt < mn)
          nl[(size_t)i * mn + cnt] = j;
        else
          overflow = 1;
        ++cnt;
      }
    }
    nn[i] = cnt;
  }
  return overflow;
}
