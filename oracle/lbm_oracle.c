/*
 * TEST INFRASTRUCTURE ONLY — the CPU restatement used as the checker.
 * Nothing in the product library links, loads or calls this file; only the
 * tests, __graft_entry__.smoke() and bench.py's cpu_baseline leg do.
 *
 * FP64 restatement of LBM-C's time step (solver.cu:10-136 with
 * collision.cu:23-503 and boundary_conditions/**), written in natural
 * population layout with two buffers.  The state is the pre-collision
 * population f_i(x, t): the reference's step t reads slot (x - t*e_i) mod L,
 * which after t in-place steps holds the post-collision value node x - e_i
 * wrote at step t-1 (solver.cu:77-94, 120-123); so step 0 collides the
 * initial populations without streaming.  Here each node collides its own
 * f_i(x, t) and pushes the result to x + e_i (periodic wrap) in the other
 * buffer.  Arithmetic follows the
 * reference's expression order so that the as-is variant is bit-identical to
 * the host-compiled reference on the paths its defects do not touch (checked
 * by tests/test_oracle_pin.py against oracle/_ref and tests/golden/).
 *
 * Differences from the reference, each selectable:
 *   - compat bits reproduce the reference's defects exactly (COMPAT_* below);
 *     without them the defects are fixed: D3Q15 M_inv = M^T D^-1,
 *     (-7/3) = -2.333.., zh_pressure_Z uses u_z, MRTPOR blends with the
 *     pre-collision opposite population;
 *   - Smagorinsky always zero-initialises q_bar (collision.cu:447 leaves it
 *     uninitialised, which is undefined behaviour);
 *   - stress-free micro BCs copy the inward populations {i : e_i.n > 0} of the
 *     interior neighbour after streaming (the reference reads unshifted slots
 *     and races with the neighbour, d2q9_sf_defs.cu:7-12, d3q15_sf_defs.cu).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define ORC_COMPAT_D3Q15_MINV_ZERO (1u << 0)
#define ORC_COMPAT_MEQ_INT_DIV (1u << 1)
#define ORC_COMPAT_ZH_Z_UX (1u << 2)
#define ORC_COMPAT_MRTPOR_INPLACE (1u << 3)

typedef struct {
  int lattice; /* 0 = D2Q9, 1 = D3Q15 */
  int length[3];
  double tau;
  double tau_mrt[15];
  double c_smag;
  int collision_type; /* 0 BGK, 1 NTPOR, 2 MRT, 3 MRTPOR */
  int forcing;
  int macro_bc;
  int micro_bc;
  unsigned compat;
} orc_config;

typedef struct {
  orc_config cfg;
  int dim, q;
  long n;
  int e[3][15];
  double w[15];
  int opp[15];
  double M[15][15];
  double Minv[15][15];
  double *f, *g; /* current / next, Q*N natural layout */
  double *geometry, *force, *u, *rho;
  int *macro, *micro;
  const double *tau_field; /* per-node relaxation time replacing Smagorinsky, or NULL */
  long step;
} orc_state;

/* ---- lattice tables: LBM-C/macros.cu:19-53 (D2Q9), :71-119 (D3Q15) ---- */

static const int E9[2][9] = {{0, 1, 0, -1, 0, 1, -1, -1, 1},
                             {0, 0, 1, 0, -1, 1, 1, -1, -1}};
static const int OPP9[9] = {0, 3, 4, 1, 2, 7, 8, 5, 6};
static const int M9[9][9] = {
    {1, 1, 1, 1, 1, 1, 1, 1, 1},      {-4, -1, -1, -1, -1, 2, 2, 2, 2},
    {4, -2, -2, -2, -2, 1, 1, 1, 1},  {0, 1, 0, -1, 0, 1, -1, -1, 1},
    {0, -2, 0, 2, 0, 1, -1, -1, 1},   {0, 0, 1, 0, -1, 1, 1, -1, -1},
    {0, 0, -2, 0, 2, 1, 1, -1, -1},   {0, 1, -1, 1, -1, 0, 0, 0, 0},
    {0, 0, 0, 0, 0, 1, -1, 1, -1}};
/* The reference's D2Q9 M^-1 is a table of decimal literals
 * (LBM-C/macros.cu:38-50); they round to slightly different doubles than
 * M^T D^-1 (e.g. -0.02777777777777779, and +-1.39e-17 where the exact entry
 * is 0), so the restatement carries the same values to stay bit-identical. */
static const double MINV9[9][9] = {
    {0.1111111111111111, -0.11111111111111112, 0.1111111111111111, 0, 0, 0, 0, 0, 0},
    {0.1111111111111111, -0.02777777777777779, -0.055555555555555566, 0.16666666666666666,
     -0.16666666666666669, 0, 0, 0.25, 0},
    {0.1111111111111111, -0.027777777777777762, -0.055555555555555539, 0,
     -1.3877787807814457e-017, 0.16666666666666666, -0.16666666666666669, -0.25, 0},
    {0.1111111111111111, -0.02777777777777779, -0.055555555555555566, -0.16666666666666666,
     0.16666666666666669, 0, 0, 0.25, 0},
    {0.1111111111111111, -0.02777777777777779, -0.055555555555555566, 0,
     1.3877787807814457e-017, -0.16666666666666666, 0.16666666666666669, -0.25, 0},
    {0.1111111111111111, 0.055555555555555552, 0.027777777777777776, 0.16666666666666666,
     0.083333333333333329, 0.16666666666666666, 0.083333333333333329, 0, 0.25},
    {0.1111111111111111, 0.055555555555555552, 0.027777777777777776, -0.16666666666666666,
     -0.083333333333333329, 0.16666666666666666, 0.083333333333333329, 0, -0.25},
    {0.1111111111111111, 0.055555555555555552, 0.027777777777777776, -0.16666666666666666,
     -0.083333333333333329, -0.16666666666666666, -0.083333333333333329, 0, 0.25},
    {0.1111111111111111, 0.055555555555555552, 0.027777777777777776, 0.16666666666666666,
     0.083333333333333329, -0.16666666666666666, -0.083333333333333329, 0, -0.25}};

static const int E15[3][15] = {
    {0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1},
    {0, 0, 0, 1, -1, 0, 0, 1, 1, -1, -1, 1, 1, -1, -1},
    {0, 0, 0, 0, 0, 1, -1, 1, 1, 1, 1, -1, -1, -1, -1}};
static const int OPP15[15] = {0, 2, 1, 4, 3, 6, 5, 14, 13, 12, 11, 10, 9, 8, 7};
static const int M15[15][15] = {
    {1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1},
    {-2, -1, -1, -1, -1, -1, -1, 1, 1, 1, 1, 1, 1, 1, 1},
    {16, -4, -4, -4, -4, -4, -4, 1, 1, 1, 1, 1, 1, 1, 1},
    {0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1},
    {0, -4, 4, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1},
    {0, 0, 0, 1, -1, 0, 0, 1, 1, -1, -1, 1, 1, -1, -1},
    {0, 0, 0, -4, 4, 0, 0, 1, 1, -1, -1, 1, 1, -1, -1},
    {0, 0, 0, 0, 0, 1, -1, 1, 1, 1, 1, -1, -1, -1, -1},
    {0, 0, 0, 0, 0, -4, 4, 1, 1, 1, 1, -1, -1, -1, -1},
    {0, 2, 2, -1, -1, -1, -1, 0, 0, 0, 0, 0, 0, 0, 0},
    {0, 0, 0, 1, 1, -1, -1, 0, 0, 0, 0, 0, 0, 0, 0},
    {0, 0, 0, 0, 0, 0, 0, 1, -1, -1, 1, 1, -1, -1, 1},
    {0, 0, 0, 0, 0, 0, 0, 1, 1, -1, -1, -1, -1, 1, 1},
    {0, 0, 0, 0, 0, 0, 0, 1, -1, 1, -1, -1, 1, -1, 1},
    {0, 0, 0, 0, 0, 0, 0, 1, -1, -1, 1, -1, 1, 1, -1}};

static void load_tables(orc_state *s) {
  memset(s->e, 0, sizeof(s->e));
  if (s->cfg.lattice == 0) {
    s->dim = 2;
    s->q = 9;
    const double w9[9] = {4.0 / 9.0, 1.0 / 9.0, 1.0 / 9.0, 1.0 / 9.0, 1.0 / 9.0,
                          1.0 / 36.0, 1.0 / 36.0, 1.0 / 36.0, 1.0 / 36.0};
    for (int i = 0; i < 9; i++) {
      s->e[0][i] = E9[0][i];
      s->e[1][i] = E9[1][i];
      s->w[i] = w9[i];
      s->opp[i] = OPP9[i];
      for (int j = 0; j < 9; j++) {
        s->M[i][j] = M9[i][j];
        s->Minv[i][j] = MINV9[i][j];
      }
    }
  } else {
    s->dim = 3;
    s->q = 15;
    for (int i = 0; i < 15; i++) {
      for (int d = 0; d < 3; d++) s->e[d][i] = E15[d][i];
      s->w[i] = i == 0 ? 2.0 / 9.0 : (i < 7 ? 1.0 / 9.0 : 1.0 / 72.0);
      s->opp[i] = OPP15[i];
      for (int j = 0; j < 15; j++) s->M[i][j] = M15[i][j];
    }
    /* M has orthogonal rows, so M^-1 = M^T D^-1 with D = diag(M M^T). */
    for (int i = 0; i < 15; i++) {
      for (int j = 0; j < 15; j++) {
        if (s->cfg.compat & ORC_COMPAT_D3Q15_MINV_ZERO) {
          s->Minv[i][j] = 0.0;
        } else {
          double norm = 0.0;
          for (int k = 0; k < 15; k++) norm += (double)(M15[j][k] * M15[j][k]);
          s->Minv[i][j] = (double)M15[j][i] / norm;
        }
      }
    }
  }
}

/* ---- per-node state, the reference's Node (data_types.cuh:45-55) ---- */
typedef struct {
  double f[15];
  double rho;
  double u[3];
  double F[3];
  double B;
  double c_smag;
  long ixd;
} node_t;

/* collision.cu:23-34 */
static double u_square(const orc_state *s, const node_t *nd) {
  double v = 0;
  for (int d = 0; d < s->dim; d++) v += nd->u[d] * nd->u[d];
  return v * 1.5;
}

/* collision.cu:36-47 */
static double e_mul_u(const orc_state *s, const node_t *nd, int i) {
  double v = 0;
  for (int d = 0; d < s->dim; d++) v += s->e[d][i] * nd->u[d];
  return v * 3.;
}

/* collision.cu:58 and its copies: rho w_i (1 + 3eu + 4.5(eu)^2 - 1.5u^2) */
static void equilibrium(const orc_state *s, const node_t *nd, double *feq) {
  const double usq = u_square(s, nd);
  for (int i = 0; i < s->q; i++) {
    const double eu = e_mul_u(s, nd, i);
    feq[i] = nd->rho * s->w[i] * (1.0 + eu + (0.5 * eu * eu) - usq);
  }
}

/* collision.cu:77 and copies: u <- u + F/(2 rho) */
static void guo_shift_velocity(const orc_state *s, node_t *nd) {
  for (int d = 0; d < s->dim; d++) nd->u[d] = nd->u[d] + (1 / (2 * nd->rho)) * nd->F[d];
}

/* collision.cu:82-99: w_i (1 - 1/2tau) [3(e_i - u) + 9 (e_i.u) e_i] . F */
static void guo_force_terms(const orc_state *s, const node_t *nd, double tau, double *ft) {
  for (int i = 0; i < s->q; i++) {
    double coeff[3];
    double dot = s->e[0][i] * nd->u[0] + s->e[1][i] * nd->u[1];
    if (s->dim > 2) dot = s->e[0][i] * nd->u[0] + s->e[1][i] * nd->u[1] + s->e[2][i] * nd->u[2];
    for (int d = 0; d < s->dim; d++)
      coeff[d] = s->w[i] * (1 - (1 / (2 * tau))) *
                 (((s->e[d][i] - nd->u[d]) * 3) + (s->e[d][i] * 9 * dot));
    ft[i] = 0;
    for (int d = 0; d < s->dim; d++) ft[i] += coeff[d] * nd->F[d];
  }
}

/* collision.cu:445-463 with q_bar zero-initialised. */
static void turbulent_viscosity(const orc_state *s, const node_t *nd, const double *feq,
                                double *tau) {
  double q_bar[3][3] = {{0}};
  double q_hat = 0.;
  for (int a = 0; a < s->dim; a++) {
    for (int b = 0; b < s->dim; b++) {
      for (int q = 0; q < s->q; q++)
        q_bar[a][b] = q_bar[a][b] + ((double)s->e[a][q] * (double)s->e[b][q] * (nd->f[q] - feq[q]));
      q_hat = q_hat + sqrt((double)2 * q_bar[a][b] * q_bar[a][b]);
    }
  }
  /* rho*POW4(1/sqrt(3)) expands textually to rho*1/sqrt(3)*1/sqrt(3)*... */
  const double r3 = sqrt((double)3);
  const double rho_pow = nd->rho * 1 / r3 * 1 / r3 * 1 / r3 * 1 / r3;
  *tau = *tau + 0.5 * (sqrt(((*tau) * (*tau)) +
                            (2 * sqrt((double)2) * (nd->c_smag * nd->c_smag) * (1 / rho_pow) * q_hat)) -
                       *tau);
}

/* collision.cu:465-503 */
static void moment_equilibrium(const orc_state *s, const node_t *nd, double *meq) {
  if (s->q == 9) {
    const double jx = nd->rho * nd->u[0];
    const double jy = nd->rho * nd->u[1];
    meq[0] = nd->rho;
    meq[1] = (-2 * nd->rho) + 3 * (jx * jx + jy * jy);
    meq[2] = nd->rho - 3 * (jx * jx + jy * jy);
    meq[3] = jx;
    meq[4] = -jx;
    meq[5] = jy;
    meq[6] = -jy;
    meq[7] = jx * jx - jy * jy;
    meq[8] = jx * jy;
  } else {
    const double jx = nd->rho * nd->u[0];
    const double jy = nd->rho * nd->u[1];
    const double jz = nd->rho * nd->u[2];
    const double c73 = (s->cfg.compat & ORC_COMPAT_MEQ_INT_DIV) ? (double)(-7 / 3) : (-7.0 / 3.0);
    meq[0] = nd->rho;
    meq[1] = (-1 * nd->rho) + (jx * jx + jy * jy + jz * jz);
    meq[2] = nd->rho - 5 * (jx * jx + jy * jy + jz * jz);
    meq[3] = jx;
    meq[4] = c73 * jx;
    meq[5] = jy;
    meq[6] = c73 * jy;
    meq[7] = jz;
    meq[8] = c73 * jz;
    meq[9] = (2 * jx * jx - (jy * jy + jz * jz));
    meq[10] = jy * jy - jz * jz;
    meq[11] = jx * jy;
    meq[12] = jy * jz;
    meq[13] = jx * jz;
    meq[14] = 0;
  }
}

/* m* = S (M f - m_eq), then acc = M^-1 m* (collision.cu:204-228). */
static void mrt_relax(const orc_state *s, const node_t *nd, double *acc) {
  double meq[15], m[15];
  moment_equilibrium(s, nd, meq);
  for (int i = 0; i < s->q; i++) {
    m[i] = 0;
    for (int j = 0; j < s->q; j++) m[i] = m[i] + s->M[i][j] * nd->f[j];
  }
  for (int i = 0; i < s->q; i++) m[i] = s->cfg.tau_mrt[i] * (m[i] - meq[i]);
  for (int i = 0; i < s->q; i++) {
    acc[i] = 0;
    for (int j = 0; j < s->q; j++) acc[i] = acc[i] + s->Minv[i][j] * m[j];
  }
}

/* collision_functions[2*type + forcing] (collision.cu:19-21), or bounceback
 * (collision.cu:423-443) when B >= 1 (solver.cu:67-72). */
static void collide(const orc_state *s, node_t *nd, double tau, int solid) {
  const int q = s->q;
  double feq[15], ft[15], tmp[15], acc[15];
  const int type = s->cfg.collision_type;
  const int forcing = s->cfg.forcing;
  if (solid) {
    for (int i = 0; i < q; i++) tmp[i] = nd->f[i];
    for (int i = 0; i < q; i++) nd->f[i] = tmp[s->opp[i]];
    nd->u[0] = 0;
    nd->u[1] = 0;
    nd->u[2] = 0;
    nd->rho = 0;
    return;
  }
  if (type == 0 || type == 1) {
    if (forcing) {
      guo_shift_velocity(s, nd);
      /* bgk_guo_collision computes force terms and equilibria in one loop;
         the values are the same when split. */
      guo_force_terms(s, nd, tau, ft);
    }
    equilibrium(s, nd, feq);
    /* A closure supplies the node's relaxation time where the reference
       would call turbulent_viscosity; the Guo terms keep tau0, as there. */
    if (s->tau_field) tau = s->tau_field[nd->ixd];
    else if (nd->c_smag > 0) turbulent_viscosity(s, nd, feq, &tau);
    if (type == 0) {
      for (int i = 0; i < q; i++) {
        if (forcing)
          nd->f[i] = nd->f[i] - (1.0 / (tau)) * (nd->f[i] - feq[i]) + ft[i];
        else
          nd->f[i] = nd->f[i] - (1.0 / (tau)) * (nd->f[i] - feq[i]);
      }
    } else {
      const double B = nd->B;
      for (int i = 0; i < q; i++) {
        const double cb = (1.0 / (tau)) * (nd->f[i] - feq[i]);
        const double cs = nd->f[s->opp[i]] - nd->f[i];
        if (forcing)
          tmp[i] = nd->f[i] - (1 - (B)) * (cb) + (B) * cs + (1 - (B)) * ft[i];
        else
          tmp[i] = nd->f[i] - (1 - (B)) * cb + (B) * cs;
      }
      for (int i = 0; i < q; i++) nd->f[i] = tmp[i];
    }
  } else {
    if (forcing) {
      guo_shift_velocity(s, nd);
      guo_force_terms(s, nd, tau, ft);
    }
    mrt_relax(s, nd, acc);
    if (type == 2) {
      for (int i = 0; i < q; i++) {
        if (forcing)
          nd->f[i] = nd->f[i] - acc[i] + ft[i];
        else
          nd->f[i] = nd->f[i] - acc[i];
      }
    } else {
      const double B = nd->B;
      double pre[15];
      for (int i = 0; i < q; i++) pre[i] = nd->f[i];
      const int inplace = (s->cfg.compat & ORC_COMPAT_MRTPOR_INPLACE) != 0;
      for (int i = 0; i < q; i++) {
        /* collision.cu:340,416 read f[opp[i]] after earlier i were updated. */
        const double fo = inplace ? nd->f[s->opp[i]] : pre[s->opp[i]];
        const double cs = fo - nd->f[i];
        if (forcing)
          nd->f[i] = nd->f[i] - (1 - (B)) * acc[i] + (1 - (B)) * ft[i] + (B) * cs;
        else
          nd->f[i] = nd->f[i] - (1 - (B)) * acc[i] + (B) * cs;
      }
    }
  }
}

/* macro_conditions[code-1] (macro_bc.cu:12-125): bit 0 ux, bit 1 uy,
 * bit 2 uz, bit 3 rho, in the table's order of codes. */
static const unsigned MACRO_MASK[16] = {0,     0x1, 0x2, 0x4, 0x3, 0x5, 0x6, 0x7,
                                        0x8,   0x9, 0xA, 0xC, 0xB, 0xD, 0xE, 0xF};

static void macro_bc(const orc_state *s, node_t *nd, int code) {
  const unsigned m = MACRO_MASK[code];
  const long n = s->n;
  if (m & 0x8) nd->rho = s->rho[nd->ixd];
  if (m & 0x1) nd->u[0] = s->u[0 * n + nd->ixd];
  if (m & 0x2) nd->u[1] = s->u[1 * n + nd->ixd];
  if ((m & 0x4) && s->dim > 2) nd->u[2] = s->u[2 * n + nd->ixd];
}

/* d2q9_zh_defs.cu:4-27 */
static void zh_d2q9(node_t *nd, int code) {
  double *f = nd->f;
  if (code == 1) {
    nd->u[0] = 1.0 - ((1.0 / nd->rho) * (f[0] + f[2] + f[4] + 2.0 * (f[3] + f[6] + f[7])));
    nd->u[1] = 0.0;
    f[1] = f[3] + ((2.0 / 3.0) * nd->rho * nd->u[0]);
    f[5] = f[7] - ((1.0 / 2.0) * (f[2] - f[4])) + ((1.0 / 6.0) * nd->rho * nd->u[0]);
    f[8] = f[6] + ((1.0 / 2.0) * (f[2] - f[4])) + ((1.0 / 6.0) * nd->rho * nd->u[0]);
  } else {
    nd->u[0] = -1.0 + ((1.0 / nd->rho) * (f[0] + f[2] + f[4] + 2.0 * (f[1] + f[5] + f[8])));
    nd->u[1] = 0.0;
    f[3] = f[1] - ((2.0 / 3.0) * nd->rho * nd->u[0]);
    f[6] = f[8] - ((1.0 / 2.0) * (f[2] - f[4])) - ((1.0 / 6.0) * nd->rho * nd->u[0]);
    f[7] = f[5] + ((1.0 / 2.0) * (f[2] - f[4])) - ((1.0 / 6.0) * nd->rho * nd->u[0]);
  }
}

/* d3q15_zh_defs.cu:4-92 */
static void zh_d3q15(const orc_state *s, node_t *nd, int code) {
  double *f = nd->f;
  const double r = nd->rho;
  switch (code) {
    case 1:
      nd->u[0] = 1.0 - ((1.0 / r) * (f[0] + f[3] + f[4] + f[5] + f[6] + 2.0 * (f[2] + f[14] + f[10] + f[12] + f[8])));
      nd->u[1] = 0.0;
      nd->u[2] = 0.0;
      f[1] = f[2] + ((2.0 / 3.0) * r * nd->u[0]);
      f[7] = f[14] + ((1.0 / 12.0) * r * nd->u[0]) - ((1.0 / 4.0) * ((-1.0) * (f[3] - f[4]) + (f[5] - f[6])));
      f[11] = f[10] + ((1.0 / 12.0) * r * nd->u[0]) - ((1.0 / 4.0) * ((-1.0) * (f[3] - f[4]) - (f[5] - f[6])));
      f[9] = f[12] + ((1.0 / 12.0) * r * nd->u[0]) - ((1.0 / 4.0) * ((f[3] - f[4]) + (f[5] - f[6])));
      f[13] = f[8] + ((1.0 / 12.0) * r * nd->u[0]) - ((1.0 / 4.0) * ((f[3] - f[4]) - (f[5] - f[6])));
      break;
    case 2:
      nd->u[0] = -1.0 + ((1.0 / r) * (f[0] + f[3] + f[4] + f[5] + f[6] + 2.0 * (f[1] + f[7] + f[11] + f[9] + f[13])));
      nd->u[1] = 0.0;
      nd->u[2] = 0.0;
      f[2] = f[1] - ((2.0 / 3.0) * r * nd->u[0]);
      f[14] = f[7] - ((1.0 / 12.0) * r * nd->u[0]) - ((1.0 / 4.0) * ((f[3] - f[4]) - (f[5] - f[6])));
      f[10] = f[11] - ((1.0 / 12.0) * r * nd->u[0]) - ((1.0 / 4.0) * ((f[3] - f[4]) + (f[5] - f[6])));
      f[12] = f[9] - ((1.0 / 12.0) * r * nd->u[0]) - ((1.0 / 4.0) * ((-1.0) * (f[3] - f[4]) + (f[5] - f[6])));
      f[8] = f[13] - ((1.0 / 12.0) * r * nd->u[0]) - ((1.0 / 4.0) * ((-1.0) * (f[3] - f[4]) - (f[5] - f[6])));
      break;
    case 3:
      nd->u[0] = 0.0;
      nd->u[1] = 1.0 - ((1.0 / r) * (f[0] + f[1] + f[2] + f[5] + f[6] + 2.0 * (f[4] + f[14] + f[10] + f[9] + f[13])));
      nd->u[2] = 0.0;
      f[3] = f[4] + ((2.0 / 3.0) * r * nd->u[1]);
      f[7] = f[14] + ((1.0 / 12.0) * r * nd->u[1]) - ((1.0 / 4.0) * ((-1.0) * (f[1] - f[2]) + (f[5] - f[6])));
      f[11] = f[10] + ((1.0 / 12.0) * r * nd->u[1]) - ((1.0 / 4.0) * ((-1.0) * (f[1] - f[2]) - (f[5] - f[6])));
      f[12] = f[9] + ((1.0 / 12.0) * r * nd->u[1]) - ((1.0 / 4.0) * ((f[1] - f[2]) - (f[5] - f[6])));
      f[8] = f[13] + ((1.0 / 12.0) * r * nd->u[1]) - ((1.0 / 4.0) * ((f[1] - f[2]) + (f[5] - f[6])));
      break;
    case 4:
      nd->u[0] = 0.0;
      nd->u[1] = -1.0 + ((1.0 / r) * (f[0] + f[1] + f[2] + f[5] + f[6] + 2.0 * (f[3] + f[7] + f[11] + f[12] + f[8])));
      nd->u[2] = 0.0;
      f[4] = f[3] - ((2.0 / 3.0) * r * nd->u[1]);
      f[14] = f[7] - ((1.0 / 12.0) * r * nd->u[1]) - ((1.0 / 4.0) * ((f[1] - f[2]) - (f[5] - f[6])));
      f[10] = f[11] - ((1.0 / 12.0) * r * nd->u[1]) - ((1.0 / 4.0) * ((f[1] - f[2]) + (f[5] - f[6])));
      f[9] = f[12] - ((1.0 / 12.0) * r * nd->u[1]) - ((1.0 / 4.0) * ((-1.0) * (f[1] - f[2]) + (f[5] - f[6])));
      f[13] = f[8] - ((1.0 / 12.0) * r * nd->u[1]) - ((1.0 / 4.0) * ((-1.0) * (f[1] - f[2]) - (f[5] - f[6])));
      break;
    case 5:
      nd->u[0] = 0.0;
      nd->u[1] = 0.0;
      nd->u[2] = 1.0 - ((1.0 / r) * (f[0] + f[1] + f[2] + f[3] + f[4] + 2.0 * (f[6] + f[14] + f[11] + f[12] + f[13])));
      f[5] = f[6] + ((2.0 / 3.0) * r * nd->u[2]);
      f[7] = f[14] + ((1.0 / 12.0) * r * nd->u[2]) - ((1.0 / 4.0) * ((-1.0) * (f[1] - f[2]) + (f[3] - f[4])));
      f[10] = f[11] + ((1.0 / 12.0) * r * nd->u[2]) - ((1.0 / 4.0) * ((f[1] - f[2]) - (f[3] - f[4])));
      f[9] = f[12] + ((1.0 / 12.0) * r * nd->u[2]) - ((1.0 / 4.0) * ((-1.0) * (f[1] - f[2]) - (f[3] - f[4])));
      f[8] = f[13] + ((1.0 / 12.0) * r * nd->u[2]) - ((1.0 / 4.0) * ((f[1] - f[2]) + (f[3] - f[4])));
      break;
    case 6: {
      nd->u[0] = 0.0;
      nd->u[1] = 0.0;
      nd->u[2] = -1.0 + ((1.0 / r) * (f[0] + f[1] + f[2] + f[3] + f[4] + 2.0 * (f[5] + f[7] + f[10] + f[9] + f[8])));
      /* d3q15_zh_defs.cu:87-91 use u[0] (zero here); the fix uses u[2]. */
      const double uz = (s->cfg.compat & ORC_COMPAT_ZH_Z_UX) ? nd->u[0] : nd->u[2];
      f[6] = f[5] - ((2.0 / 3.0) * r * uz);
      f[14] = f[7] - ((1.0 / 12.0) * r * uz) - ((1.0 / 4.0) * ((f[1] - f[2]) - (f[3] - f[4])));
      f[11] = f[10] - ((1.0 / 12.0) * r * uz) - ((1.0 / 4.0) * ((-1.0) * (f[1] - f[2]) + (f[3] - f[4])));
      f[12] = f[9] - ((1.0 / 12.0) * r * uz) - ((1.0 / 4.0) * ((f[1] - f[2]) + (f[3] - f[4])));
      f[13] = f[8] - ((1.0 / 12.0) * r * uz) - ((1.0 / 4.0) * ((-1.0) * (f[1] - f[2]) - (f[3] - f[4])));
      break;
    }
    default:
      break;
  }
}

static long wrap(long v, long L) {
  v %= L;
  return v < 0 ? v + L : v;
}

static long node_index(const orc_state *s, const long *c) {
  const int *L = s->cfg.length;
  return c[0] + L[0] * (c[1] + (long)L[1] * c[2]);
}

/* Pre-collision (post-streaming) population i of node c. */
static double pulled(const orc_state *s, const long *c, int i) {
  return s->f[(long)i * s->n + node_index(s, c)];
}

/* Stress-free copy: face normal axis/sign per code (x, X, y, Y, z, Z). */
static void sf_copy(const orc_state *s, node_t *nd, const long *c, int which) {
  const int axis = which / 2;
  const int inward = (which % 2 == 0) ? 1 : -1; /* sf_x at the low face copies from x+1 */
  long nb[3] = {c[0], c[1], c[2]};
  nb[axis] = wrap(nb[axis] + inward, s->cfg.length[axis]);
  for (int i = 0; i < s->q; i++)
    if (s->e[axis][i] * inward > 0) nd->f[i] = pulled(s, nb, i);
}

static void micro_bc(const orc_state *s, node_t *nd, const long *c, int code) {
  if (s->q == 9) {
    if (code == 1 || code == 2) zh_d2q9(nd, code);
    else if (code >= 5 && code <= 8) sf_copy(s, nd, c, code - 5);
  } else {
    if (code >= 1 && code <= 6) zh_d3q15(s, nd, code);
    else if (code >= 7 && code <= 12) sf_copy(s, nd, c, code - 7);
  }
}

/* ---------------------------- public API ---------------------------- */

orc_state *orc_create(const orc_config *cfg, const double *geometry, const double *force,
                      const int *macro, const int *micro, const double *u, const double *rho,
                      const double *f_init) {
  orc_state *s = (orc_state *)calloc(1, sizeof(orc_state));
  s->cfg = *cfg;
  load_tables(s);
  if (s->dim == 2) s->cfg.length[2] = 1;
  s->n = (long)s->cfg.length[0] * s->cfg.length[1] * s->cfg.length[2];
  const long n = s->n;
  s->f = (double *)malloc(sizeof(double) * n * s->q);
  s->g = (double *)malloc(sizeof(double) * n * s->q);
  s->geometry = (double *)calloc(n, sizeof(double));
  s->force = (double *)calloc(3 * n, sizeof(double));
  s->u = (double *)calloc(3 * n, sizeof(double));
  s->rho = (double *)calloc(n, sizeof(double));
  s->macro = (int *)calloc(n, sizeof(int));
  s->micro = (int *)calloc(n, sizeof(int));
  for (int i = 0; i < s->q; i++)
    for (long k = 0; k < n; k++) s->f[i * n + k] = f_init ? f_init[i * n + k] : 1.0 * s->w[i];
  if (geometry) memcpy(s->geometry, geometry, sizeof(double) * n);
  if (force) memcpy(s->force, force, sizeof(double) * n * s->dim);
  if (u) memcpy(s->u, u, sizeof(double) * n * s->dim);
  if (rho) memcpy(s->rho, rho, sizeof(double) * n);
  if (macro) memcpy(s->macro, macro, sizeof(int) * n);
  if (micro) memcpy(s->micro, micro, sizeof(int) * n);
  return s;
}

static void step_node(orc_state *s, long k, int store) {
  const int *L = s->cfg.length;
  const long n = s->n;
  const long c[3] = {k % L[0], (k / L[0]) % L[1], k / ((long)L[0] * L[1])};
  node_t nd;
  memset(&nd, 0, sizeof(nd));
  nd.ixd = k;
  nd.c_smag = s->cfg.c_smag;
  double tau = s->cfg.tau;
  int macro = s->cfg.macro_bc ? s->macro[k] : 0;
  int micro = s->cfg.micro_bc ? s->micro[k] : 0;
  if (s->cfg.forcing)
    for (int d = 0; d < s->dim; d++) nd.F[d] = s->force[d * n + k];
  nd.B = s->geometry[k];
  const int solid = nd.B >= 1;
  if (solid) {
    macro = 0;
    micro = 0;
  }
  /* solver.cu:75-108: load, rho = sum f, u = sum e f / rho */
  for (int i = 0; i < s->q; i++) {
    nd.f[i] = pulled(s, c, i);
    nd.rho += nd.f[i];
    for (int d = 0; d < s->dim; d++) nd.u[d] += s->e[d][i] * nd.f[i];
  }
  for (int d = 0; d < s->dim; d++) nd.u[d] = nd.u[d] / nd.rho;
  if (macro > 0) macro_bc(s, &nd, macro);
  if (micro > 0) micro_bc(s, &nd, c, micro);
  collide(s, &nd, tau, solid);
  for (int i = 0; i < s->q; i++) {
    long dst[3] = {0, 0, 0};
    for (int d = 0; d < s->dim; d++) dst[d] = wrap(c[d] + s->e[d][i], s->cfg.length[d]);
    s->g[(long)i * n + node_index(s, dst)] = nd.f[i];
  }
  if (store) {
    for (int d = 0; d < s->dim; d++) s->u[d * n + k] = nd.u[d];
    s->rho[k] = nd.rho;
  }
}

void orc_run(orc_state *s, int nsteps, int store_last) {
  for (int step = 0; step < nsteps; step++) {
    const int store = store_last && step == nsteps - 1;
#pragma omp parallel for schedule(static)
    for (long k = 0; k < s->n; k++) step_node(s, k, store);
    double *t = s->f;
    s->f = s->g;
    s->g = t;
    s->step++;
  }
}

void orc_get_f(const orc_state *s, double *out) { memcpy(out, s->f, sizeof(double) * s->n * s->q); }

void orc_get_macros(const orc_state *s, double *rho, double *u) {
  memcpy(rho, s->rho, sizeof(double) * s->n);
  memcpy(u, s->u, sizeof(double) * s->n * s->dim);
}

void orc_tables(const orc_state *s, int *e, double *w, int *opp, double *M, double *Minv) {
  for (int d = 0; d < s->dim; d++)
    for (int i = 0; i < s->q; i++) e[d * s->q + i] = s->e[d][i];
  for (int i = 0; i < s->q; i++) {
    w[i] = s->w[i];
    opp[i] = s->opp[i];
    for (int j = 0; j < s->q; j++) {
      M[i * s->q + j] = s->M[i][j];
      Minv[i * s->q + j] = s->Minv[i][j];
    }
  }
}

/* Equilibrium populations for an initial (rho, u) field: Q*N natural layout. */
void orc_equilibrium_field(const orc_state *s, const double *rho, const double *u, double *out) {
  const long n = s->n;
  for (long k = 0; k < n; k++) {
    node_t nd;
    memset(&nd, 0, sizeof(nd));
    nd.rho = rho[k];
    for (int d = 0; d < s->dim; d++) nd.u[d] = u[d * n + k];
    double feq[15];
    equilibrium(s, &nd, feq);
    for (int i = 0; i < s->q; i++) out[i * n + k] = feq[i];
  }
}

/* Per-node relaxation times for the next steps (NULL restores tau/Smagorinsky);
   the caller keeps the array alive. */
void orc_set_tau_field(orc_state *s, const double *tau) { s->tau_field = tau; }

void orc_destroy(orc_state *s) {
  if (!s) return;
  free(s->f);
  free(s->g);
  free(s->geometry);
  free(s->force);
  free(s->u);
  free(s->rho);
  free(s->macro);
  free(s->micro);
  free(s);
}
