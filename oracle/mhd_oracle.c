/* CPU restatement of the reference's explicit multi-fluid Hall-MHD step
 * (MercurySolver::StepOnce, Z4_Mercury/src/MercurySolver_Driver.cpp:21-61)
 * for ONE periodic block.  THIS IS TEST INFRASTRUCTURE (the oracle): only the
 * parity tests, the smoke check and the CPU-baseline leg of the benchmark call
 * it, to check results against it.  The product never links it.
 *
 * Every routine follows the reference function named in its comment, in the
 * reference's loop and operation order, in FP64, so that the restatement is
 * pinned to the reference build (oracle/_ref) to roundoff.
 *
 * Storage is the reference's own FieldBlock layout (include/3_field/FieldArray.h:
 * 126-128,177): AoS, offset = ((i-lo0)*e1 + (j-lo1))*e2*nc + (k-lo2)*nc + m,
 * k fastest.  Index space is FieldBlock's: owned DOFs are [0, n + stagger) per
 * axis (include/3_field/FieldBlock.h:34-35), ghosts outside.
 *
 * Synchronisation on a single periodic block follows the rule measured from
 * the reference with unique codes (Z0_NULL/test/halo_comm method):
 *   halo:  every ghost DOF copies the DOF reached by wrapping each out-of-range
 *          index by +-n (cell axes: mod n; node axes: the alias layer n is an
 *          owned DOF and is kept); Corner1D groups fill only ghosts that are
 *          out of range along exactly one axis;
 *   owner: owned alias DOFs (a node-axis index equal to n) then take the value
 *          of their owner (index 0); halo copies see the pre-owner values.
 * The net map is applied from a snapshot, as the reference's staged exchange
 * composes to.
 */
#include <math.h>
#include <stddef.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef struct {
  double *p;
  int lo[3], hi[3], nc;
} ofld;

enum { LOC_CELL = 0, LOC_FXI, LOC_FET, LOC_FZE, LOC_EXI, LOC_EET, LOC_EZE };
static const int kStag[7][3] = {{0, 0, 0}, {1, 0, 0}, {0, 1, 0}, {0, 0, 1}, {0, 1, 1}, {1, 0, 1}, {1, 1, 0}};

typedef struct {
  /* physical constants, as calc_physical_constant (Z4_Mercury/src/physics/MercurySolver_Tools.cpp:3-48) */
  double gamma, M_H, M_Na, M_ref, T_ref, L_ref, U_ref, B_ref, n_ref, rho_ref, m_Na, k_Boltz, q_e, mu0;
  double state_coeff_H, state_coeff_Na, CFL, hall_coef, momentum_induce_coeff, momentum_hall_coeff, inver_MA2;
  double ne_hall_floor;
  int ambipolar;
  int n;  /* cells per axis (cube block) */
  /* state */
  ofld UH, UN, Bx, By, Bz;
  /* derived */
  ofld PVH, PVN, Up, Bc, Bic, Jc, Jx, Jy, Jz;
  /* work */
  ofld RH, RN, Fx, Fy, Fz, RBx, RBy, RBz, Ex, Ey, Ez, Hx, Hy, Hz, EFx, EFy, EFz, Ehc, beta;
  /* static */
  ofld Jac, JDx, JDy, JDz, Ax, Ay, Az, dlx, dly, dlz, drx, dry, drz, bfx, bfy, bfz, alx, aly, alz, WB, WJ;
  ofld Bax, Bay, Baz, Photo, cx, cy, cz, tpx, tpy, tpz;
  double dt, time;
  long step;
} octx;

static inline double *A(const ofld *f, int i, int j, int k, int m) {
  const long e1 = f->hi[1] - f->lo[1], e2 = f->hi[2] - f->lo[2];
  return f->p + ((((long)(i - f->lo[0]) * e1 + (j - f->lo[1])) * e2 + (k - f->lo[2])) * f->nc + m);
}
#define V(f, i, j, k, m) (*A(&(f), (i), (j), (k), (m)))

/* std::max / std::min semantics (first argument wins ties, incl. signed zeros) */
static inline double dmax(double a, double b) { return (a < b) ? b : a; }
static inline double dmin(double a, double b) { return (b < a) ? b : a; }

/* inner (owned) range of a field: [0, hi - g) with g = -lo (FieldBlock.h:34-35) */
static inline int ihi(const ofld *f, int a) { return f->hi[a] + f->lo[a]; }

/* ----------------------------------------------------------------- sync */
static void sync_periodic(ofld *f, int loc, int corner1d, int n) {
  const int *st = kStag[loc];
  const long tot = (long)(f->hi[0] - f->lo[0]) * (f->hi[1] - f->lo[1]) * (f->hi[2] - f->lo[2]) * f->nc;
  double *snap = (double *)malloc(sizeof(double) * tot);
  memcpy(snap, f->p, sizeof(double) * tot);
  ofld s = *f;
  s.p = snap;
  for (int i = f->lo[0]; i < f->hi[0]; ++i)
    for (int j = f->lo[1]; j < f->hi[1]; ++j)
      for (int k = f->lo[2]; k < f->hi[2]; ++k) {
        int idx[3] = {i, j, k}, src[3];
        int nout = 0;
        for (int a = 0; a < 3; ++a) nout += !(idx[a] >= 0 && idx[a] < n + st[a]);
        if (nout == 0) {
          int alias = 0;
          for (int a = 0; a < 3; ++a) {
            src[a] = (st[a] && idx[a] == n) ? 0 : idx[a];
            alias |= (st[a] && idx[a] == n);
          }
          if (!alias) continue;
        } else {
          if (corner1d && nout > 1) continue;
          for (int a = 0; a < 3; ++a) {
            int v = idx[a];
            if (st[a]) {
              if (v < 0) v += n;
              else if (v > n) v -= n;
            } else {
              v = ((v % n) + n) % n;
            }
            src[a] = v;
          }
        }
        for (int m = 0; m < f->nc; ++m) *A(f, i, j, k, m) = *A(&s, src[0], src[1], src[2], m);
      }
  free(snap);
}

/* ReduceEdgeAliasCandidatesToOwners_ (Z4_Mercury/src/physics/MercurySolver_Current.cpp:3-57)
 * on a periodic cube: each edge class with more than one member is written to
 * its owner (all node indices in [0, n)) as the member sum, accumulated in the
 * class's member order (lexicographic (i, j, k) of the aliases), divided by the
 * member count.  Orientation signs of a periodic class are equal and cancel
 * exactly. */
static void alias_reduce_edges(ofld *E, int loc, int n) {
  const int *st = kStag[loc];
  const int ext[3] = {n + st[0], n + st[1], n + st[2]};
  for (int i = 0; i < ext[0]; ++i)
    for (int j = 0; j < ext[1]; ++j)
      for (int k = 0; k < ext[2]; ++k) {
        const int idx[3] = {i, j, k};
        int ok = 1, dup = 0;
        for (int a = 0; a < 3; ++a) {
          if (st[a] && idx[a] == n) ok = 0;
          if (st[a] && idx[a] == 0) dup = 1;
        }
        if (!ok || !dup) continue;
        /* enumerate members lexicographically: each boundary node axis takes {0, n} */
        int na = 0, axes[3];
        for (int a = 0; a < 3; ++a)
          if (st[a] && idx[a] == 0) axes[na++] = a;
        const int count = 1 << na;
        double sum = 0.0;
        for (int c = 0; c < count; ++c) {
          int p[3] = {i, j, k};
          for (int b = 0; b < na; ++b)
            if (c & (1 << (na - 1 - b))) p[axes[b]] = n;
          sum += V(*E, p[0], p[1], p[2], 0);
        }
        V(*E, i, j, k, 0) = sum / (double)count;
      }
}

/* ----------------------------------------------------------------- tools */
typedef struct {
  double nH, nNa, ne_true, ne_eff, chiH, chiNa, wH, wNa;
} numinfo;

/* Hall_Num_Limiter (Z4_Mercury/src/physics/MercurySolver_Tools.cpp:111-157) */
static numinfo num_limiter(const octx *c, double rhoH, double rhoNa) {
  numinfo d;
  const double rH = dmax(rhoH, 0.0), rN = dmax(rhoNa, 0.0);
  d.nH = rH / c->M_H * c->M_ref;
  d.nNa = rN / c->M_Na * c->M_ref;
  d.ne_true = d.nH + d.nNa;
  d.ne_eff = sqrt(d.ne_true * d.ne_true + c->ne_hall_floor * c->ne_hall_floor);
  if (d.ne_true > 1.0e-300) {
    d.chiH = d.nH / d.ne_true;
    d.chiNa = d.nNa / d.ne_true;
  } else {
    d.chiH = 1.0;
    d.chiNa = 0.0;
  }
  d.wH = d.nH / d.ne_eff;
  d.wNa = d.nNa / d.ne_eff;
  return d;
}

/* calc_PV (Tools.cpp:159-213): all allocated points including ghosts */
static void calc_pv(octx *c) {
  const ofld *Us[2] = {&c->UH, &c->UN};
  ofld *Ps[2] = {&c->PVH, &c->PVN};
  const double coeff[2] = {c->state_coeff_H, c->state_coeff_Na};
  for (int s = 0; s < 2; ++s) {
    const ofld *U = Us[s];
    ofld *P = Ps[s];
    for (int i = P->lo[0]; i < P->hi[0]; ++i)
      for (int j = P->lo[1]; j < P->hi[1]; ++j)
        for (int k = P->lo[2]; k < P->hi[2]; ++k) {
          const double rho = dmax(V(*U, i, j, k, 0), 1e-12);
          const double u = V(*U, i, j, k, 1) / rho, v = V(*U, i, j, k, 2) / rho, w = V(*U, i, j, k, 3) / rho;
          const double E = V(*U, i, j, k, 4);
          const double ke = 0.5 * rho * (u * u + v * v + w * w);
          double eint = E - ke;
          if (eint < 0.0) eint = 0.0;
          double p = (c->gamma - 1.0) * eint;
          p = dmax(p, 1e-12);
          const double T = p / (rho * coeff[s]);
          V(*P, i, j, k, 0) = u;
          V(*P, i, j, k, 1) = v;
          V(*P, i, j, k, 2) = w;
          V(*P, i, j, k, 3) = p;
          V(*P, i, j, k, 4) = T;
        }
  }
}

/* calc_Uplus (Tools.cpp:215-301) */
static void calc_uplus(octx *c) {
  ofld *Up = &c->Up;
  for (int i = Up->lo[0]; i < Up->hi[0]; ++i)
    for (int j = Up->lo[1]; j < Up->hi[1]; ++j)
      for (int k = Up->lo[2]; k < Up->hi[2]; ++k) {
        const double rH = dmax(V(c->UH, i, j, k, 0), 0.0), rN = dmax(V(c->UN, i, j, k, 0), 0.0);
        const double uH = rH > 1e-20 ? V(c->PVH, i, j, k, 0) : 0.0;
        const double vH = rH > 1e-20 ? V(c->PVH, i, j, k, 1) : 0.0;
        const double wH = rH > 1e-20 ? V(c->PVH, i, j, k, 2) : 0.0;
        const double uN = rN > 1e-20 ? V(c->PVN, i, j, k, 0) : 0.0;
        const double vN = rN > 1e-20 ? V(c->PVN, i, j, k, 1) : 0.0;
        const double wN = rN > 1e-20 ? V(c->PVN, i, j, k, 2) : 0.0;
        const numinfo d = num_limiter(c, rH, rN);
        V(*Up, i, j, k, 0) = d.chiH * uH + d.chiNa * uN;
        V(*Up, i, j, k, 1) = d.chiH * vH + d.chiNa * vN;
        V(*Up, i, j, k, 2) = d.chiH * wH + d.chiNa * wN;
      }
}

/* calc_Bcell (Z4_Mercury/src/physics/MercurySolver_MagneticCell.cpp:3-90) + Sync("B_cell") */
static void calc_bcell(octx *c) {
  const int n = c->n;
  for (int i = 0; i < ihi(&c->Bc, 0); ++i)
    for (int j = 0; j < ihi(&c->Bc, 1); ++j)
      for (int k = 0; k < ihi(&c->Bc, 2); ++k) {
        const double pt[6] = {-V(c->Bx, i, j, k, 0) - V(c->Bax, i, j, k, 0), V(c->Bx, i + 1, j, k, 0) + V(c->Bax, i + 1, j, k, 0),
                              -V(c->By, i, j, k, 0) - V(c->Bay, i, j, k, 0), V(c->By, i, j + 1, k, 0) + V(c->Bay, i, j + 1, k, 0),
                              -V(c->Bz, i, j, k, 0) - V(c->Baz, i, j, k, 0), V(c->Bz, i, j, k + 1, 0) + V(c->Baz, i, j, k + 1, 0)};
        const double pi_[6] = {-V(c->Bx, i, j, k, 0), V(c->Bx, i + 1, j, k, 0), -V(c->By, i, j, k, 0),
                               V(c->By, i, j + 1, k, 0), -V(c->Bz, i, j, k, 0), V(c->Bz, i, j, k + 1, 0)};
        double bxt = 0, byt = 0, bzt = 0, bxi = 0, byi = 0, bzi = 0;
        for (int q = 0; q < 6; ++q) {
          const double wx = V(c->WB, i, j, k, q), wy = V(c->WB, i, j, k, 6 + q), wz = V(c->WB, i, j, k, 12 + q);
          bxt += wx * pt[q];
          byt += wy * pt[q];
          bzt += wz * pt[q];
          bxi += wx * pi_[q];
          byi += wy * pi_[q];
          bzi += wz * pi_[q];
        }
        V(c->Bc, i, j, k, 0) = bxt;
        V(c->Bc, i, j, k, 1) = byt;
        V(c->Bc, i, j, k, 2) = bzt;
        V(c->Bic, i, j, k, 0) = bxi;
        V(c->Bic, i, j, k, 1) = byi;
        V(c->Bic, i, j, k, 2) = bzi;
      }
  sync_periodic(&c->Bc, LOC_CELL, 0, n);
  sync_periodic(&c->Bic, LOC_CELL, 0, n);
}

/* CTOperators::CurlAdjFaceToEdge (Z4_Mercury/src/operators/CTOperators.cpp:59-110) then
 * Calc_J_Edge (Z4_Mercury/src/physics/MercurySolver_Current.cpp:140-201) */
static void calc_j_edge(octx *c) {
  const int n = c->n;
  for (int i = 0; i < ihi(&c->Jx, 0); ++i)
    for (int j = 0; j < ihi(&c->Jx, 1); ++j)
      for (int k = 0; k < ihi(&c->Jx, 2); ++k)
        V(c->Jx, i, j, k, 0) = ((V(c->bfy, i, j, k - 1, 0) * V(c->By, i, j, k - 1, 0) - V(c->bfy, i, j, k, 0) * V(c->By, i, j, k, 0)) +
                                (V(c->bfz, i, j, k, 0) * V(c->Bz, i, j, k, 0) - V(c->bfz, i, j - 1, k, 0) * V(c->Bz, i, j - 1, k, 0))) * 1.0;
  for (int i = 0; i < ihi(&c->Jy, 0); ++i)
    for (int j = 0; j < ihi(&c->Jy, 1); ++j)
      for (int k = 0; k < ihi(&c->Jy, 2); ++k)
        V(c->Jy, i, j, k, 0) = ((V(c->bfx, i, j, k, 0) * V(c->Bx, i, j, k, 0) - V(c->bfx, i, j, k - 1, 0) * V(c->Bx, i, j, k - 1, 0)) +
                                (V(c->bfz, i - 1, j, k, 0) * V(c->Bz, i - 1, j, k, 0) - V(c->bfz, i, j, k, 0) * V(c->Bz, i, j, k, 0))) * 1.0;
  for (int i = 0; i < ihi(&c->Jz, 0); ++i)
    for (int j = 0; j < ihi(&c->Jz, 1); ++j)
      for (int k = 0; k < ihi(&c->Jz, 2); ++k)
        V(c->Jz, i, j, k, 0) = ((V(c->bfx, i, j - 1, k, 0) * V(c->Bx, i, j - 1, k, 0) - V(c->bfx, i, j, k, 0) * V(c->Bx, i, j, k, 0)) +
                                (V(c->bfy, i, j, k, 0) * V(c->By, i, j, k, 0) - V(c->bfy, i - 1, j, k, 0) * V(c->By, i - 1, j, k, 0))) * 1.0;
  ofld *J[3] = {&c->Jx, &c->Jy, &c->Jz};
  const ofld *al[3] = {&c->alx, &c->aly, &c->alz};
  for (int a = 0; a < 3; ++a)
    for (int i = 0; i < ihi(J[a], 0); ++i)
      for (int j = 0; j < ihi(J[a], 1); ++j)
        for (int k = 0; k < ihi(J[a], 2); ++k) *A(J[a], i, j, k, 0) *= *A(al[a], i, j, k, 0);
  alias_reduce_edges(&c->Jx, LOC_EXI, n);
  alias_reduce_edges(&c->Jy, LOC_EET, n);
  alias_reduce_edges(&c->Jz, LOC_EZE, n);
  sync_periodic(&c->Jx, LOC_EXI, 0, n);
  sync_periodic(&c->Jy, LOC_EET, 0, n);
  sync_periodic(&c->Jz, LOC_EZE, 0, n);
}

/* calc_Jcell (Current.cpp:203-243) + Sync("J_cell"); no Pole patches on the cube */
static void calc_jcell(octx *c) {
  for (int i = 0; i < ihi(&c->Jc, 0); ++i)
    for (int j = 0; j < ihi(&c->Jc, 1); ++j)
      for (int k = 0; k < ihi(&c->Jc, 2); ++k) {
        const double s[12] = {V(c->Jx, i, j, k, 0),     V(c->Jx, i, j + 1, k, 0),     V(c->Jx, i, j, k + 1, 0),
                              V(c->Jx, i, j + 1, k + 1, 0), V(c->Jy, i, j, k, 0),     V(c->Jy, i + 1, j, k, 0),
                              V(c->Jy, i, j, k + 1, 0),     V(c->Jy, i + 1, j, k + 1, 0), V(c->Jz, i, j, k, 0),
                              V(c->Jz, i + 1, j, k, 0),     V(c->Jz, i, j + 1, k, 0),     V(c->Jz, i + 1, j + 1, k, 0)};
        double jx = 0, jy = 0, jz = 0;
        for (int q = 0; q < 12; ++q) {
          jx += V(c->WJ, i, j, k, q) * s[q];
          jy += V(c->WJ, i, j, k, 12 + q) * s[q];
          jz += V(c->WJ, i, j, k, 24 + q) * s[q];
        }
        V(c->Jc, i, j, k, 0) = jx;
        V(c->Jc, i, j, k, 1) = jy;
        V(c->Jc, i, j, k, 2) = jz;
      }
  sync_periodic(&c->Jc, LOC_CELL, 0, c->n);
}

/* UpdateDerivedFields_ (Tools.cpp:309-321) */
void oracle_update_derived(octx *c) {
  calc_bcell(c);
  calc_j_edge(c);
  calc_jcell(c);
  calc_pv(c);
  calc_uplus(c);
}

/* ----------------------------------------------------------------- step pieces */
/* Compute_Timestep (Z4_Mercury/src/physics/MercurySolver_Timestep.cpp:8-141) */
static double fast_cf(double cs2, double vA2, double vAn2) {
  const double term = cs2 + vA2;
  double disc = term * term - 4.0 * cs2 * vAn2;
  if (disc < 0.0) disc = 0.0;
  return sqrt(0.5 * (term + sqrt(disc)));
}
static double face_term(const octx *c, double ax, double ay, double az, int outward_plus, double ux, double uy, double uz,
                        double Bx, double By, double Bz, double B2, double rho, double cs2) {
  const double An = sqrt(ax * ax + ay * ay + az * az);
  if (An <= 0.0) return 0.0;
  double nx = ax / An, ny = ay / An, nz = az / An;
  if (!outward_plus) {
    nx = -nx;
    ny = -ny;
    nz = -nz;
  }
  const double un = ux * nx + uy * ny + uz * nz;
  const double Bn = Bx * nx + By * ny + Bz * nz;
  const double vA2 = c->inver_MA2 * B2 / rho;
  const double vAn2 = c->inver_MA2 * (Bn * Bn) / rho;
  const double cf = fast_cf(cs2, vA2, vAn2);
  return (fabs(un) + cf) * An;
}
static double compute_timestep(const octx *c) {
  double dtl = 1e100;
  const ofld *Us[2] = {&c->UH, &c->UN};
  for (int s = 0; s < 2; ++s) {
    const ofld *U = Us[s];
    for (int i = 0; i < ihi(&c->Jac, 0); ++i)
      for (int j = 0; j < ihi(&c->Jac, 1); ++j)
        for (int k = 0; k < ihi(&c->Jac, 2); ++k) {
          const double Vol = fabs(V(c->Jac, i, j, k, 0));
          if (Vol <= 0.0) continue;
          const double rho = dmax(V(*U, i, j, k, 0), 1e-2);
          const double ux = V(*U, i, j, k, 1) / rho, uy = V(*U, i, j, k, 2) / rho, uz = V(*U, i, j, k, 3) / rho;
          const double E = V(*U, i, j, k, 4);
          const double ke = 0.5 * rho * (ux * ux + uy * uy + uz * uz);
          const double p = (c->gamma - 1.0) * (E - ke);
          const double cs2 = c->gamma * p / rho;
          const double Bx = V(c->Bc, i, j, k, 0), By = V(c->Bc, i, j, k, 1), Bz = V(c->Bc, i, j, k, 2);
          const double B2 = Bx * Bx + By * By + Bz * Bz;
          double den = 0.0;
          den += face_term(c, V(c->JDx, i, j, k, 0), V(c->JDx, i, j, k, 1), V(c->JDx, i, j, k, 2), 0, ux, uy, uz, Bx, By, Bz, B2, rho, cs2);
          den += face_term(c, V(c->JDx, i + 1, j, k, 0), V(c->JDx, i + 1, j, k, 1), V(c->JDx, i + 1, j, k, 2), 1, ux, uy, uz, Bx, By, Bz, B2, rho, cs2);
          den += face_term(c, V(c->JDy, i, j, k, 0), V(c->JDy, i, j, k, 1), V(c->JDy, i, j, k, 2), 0, ux, uy, uz, Bx, By, Bz, B2, rho, cs2);
          den += face_term(c, V(c->JDy, i, j + 1, k, 0), V(c->JDy, i, j + 1, k, 1), V(c->JDy, i, j + 1, k, 2), 1, ux, uy, uz, Bx, By, Bz, B2, rho, cs2);
          den += face_term(c, V(c->JDz, i, j, k, 0), V(c->JDz, i, j, k, 1), V(c->JDz, i, j, k, 2), 0, ux, uy, uz, Bx, By, Bz, B2, rho, cs2);
          den += face_term(c, V(c->JDz, i, j, k + 1, 0), V(c->JDz, i, j, k + 1, 1), V(c->JDz, i, j, k + 1, 2), 1, ux, uy, uz, Bx, By, Bz, B2, rho, cs2);
          if (den > 0.0) dtl = dmin(dtl, c->CFL * Vol / den);
        }
  }
  return dtl;
}

/* Scheme_U_ (Z4_Mercury/src/physics/MercurySolver_FluidRHS.cpp:3-202) */
static void rusanov_face(const octx *c, const double *met, int dir, const ofld *PV, const ofld *U, int i, int j, int k, double *out) {
  const double k1 = met[0], k2 = met[1], k3 = met[2];
  int iL = i, jL = j, kL = k;
  if (dir == 0) iL = i - 1;
  if (dir == 1) jL = j - 1;
  if (dir == 2) kL = k - 1;
  const double g = c->gamma;
  const double rhoL = V(*U, iL, jL, kL, 0), uL = V(*PV, iL, jL, kL, 0), vL = V(*PV, iL, jL, kL, 1), wL = V(*PV, iL, jL, kL, 2),
               pL = V(*PV, iL, jL, kL, 3);
  const double rhoR = V(*U, i, j, k, 0), uR = V(*PV, i, j, k, 0), vR = V(*PV, i, j, k, 1), wR = V(*PV, i, j, k, 2),
               pR = V(*PV, i, j, k, 3);
  double UL[5], UR[5];
  UL[0] = rhoL;
  UL[1] = rhoL * uL;
  UL[2] = rhoL * vL;
  UL[3] = rhoL * wL;
  UL[4] = pL / (g - 1.0) + 0.5 * rhoL * (uL * uL + vL * vL + wL * wL);
  UR[0] = rhoR;
  UR[1] = rhoR * uR;
  UR[2] = rhoR * vR;
  UR[3] = rhoR * wR;
  UR[4] = pR / (g - 1.0) + 0.5 * rhoR * (uR * uR + vR * vR + wR * wR);
  const double kk = k1 * k1 + k2 * k2 + k3 * k3;
  const double uvwL = k1 * uL + k2 * vL + k3 * wL, uvwR = k1 * uR + k2 * vR + k3 * wR;
  const double cL = sqrt(dmax(0.0, g * pL / dmax(rhoL, 1e-30))), cR = sqrt(dmax(0.0, g * pR / dmax(rhoR, 1e-30)));
  const double radL = fabs(uvwL) + cL * sqrt(kk), radR = fabs(uvwR) + cR * sqrt(kk);
  const double rad = dmax(radL, radR);
  double FL[5], FR[5];
  const double reL = pL / (g - 1.0) + 0.5 * rhoL * (uL * uL + vL * vL + wL * wL);
  const double reR = pR / (g - 1.0) + 0.5 * rhoR * (uR * uR + vR * vR + wR * wR);
  FL[0] = rhoL * uvwL;
  FL[1] = rhoL * uvwL * uL + k1 * pL;
  FL[2] = rhoL * uvwL * vL + k2 * pL;
  FL[3] = rhoL * uvwL * wL + k3 * pL;
  FL[4] = uvwL * (reL + pL);
  FR[0] = rhoR * uvwR;
  FR[1] = rhoR * uvwR * uR + k1 * pR;
  FR[2] = rhoR * uvwR * vR + k2 * pR;
  FR[3] = rhoR * uvwR * wR + k3 * pR;
  FR[4] = uvwR * (reR + pR);
  for (int m = 0; m < 5; ++m) out[m] = 0.5 * (FL[m] + FR[m]) - 0.5 * rad * (UR[m] - UL[m]);
}
static void scheme_u(octx *c) {
  const ofld *Us[2] = {&c->UH, &c->UN}, *Ps[2] = {&c->PVH, &c->PVN};
  ofld *Rs[2] = {&c->RH, &c->RN};
  ofld *F[3] = {&c->Fx, &c->Fy, &c->Fz};
  const ofld *M[3] = {&c->JDx, &c->JDy, &c->JDz};
  for (int s = 0; s < 2; ++s) {
    for (int d = 0; d < 3; ++d)
      for (int i = 0; i < ihi(F[d], 0); ++i)
        for (int j = 0; j < ihi(F[d], 1); ++j)
          for (int k = 0; k < ihi(F[d], 2); ++k) {
            const double met[3] = {*A(M[d], i, j, k, 0), *A(M[d], i, j, k, 1), *A(M[d], i, j, k, 2)};
            double fl[5];
            rusanov_face(c, met, d, Ps[s], Us[s], i, j, k, fl);
            for (int m = 0; m < 5; ++m) *A(F[d], i, j, k, m) = fl[m];
          }
    ofld *R = Rs[s];
    for (int i = 0; i < ihi(R, 0); ++i)
      for (int j = 0; j < ihi(R, 1); ++j)
        for (int k = 0; k < ihi(R, 2); ++k) {
          const double invJ = 1.0 / V(c->Jac, i, j, k, 0);
          for (int m = 0; m < 5; ++m) {
            *A(R, i, j, k, m) -= (V(c->Fx, i + 1, j, k, m) - V(c->Fx, i, j, k, m)) * invJ;
            *A(R, i, j, k, m) -= (V(c->Fy, i, j + 1, k, m) - V(c->Fy, i, j, k, m)) * invJ;
            *A(R, i, j, k, m) -= (V(c->Fz, i, j, k + 1, m) - V(c->Fz, i, j, k, m)) * invJ;
          }
        }
  }
}

/* AddSourceToRHS_Fluid (FluidRHS.cpp:206-527) */
static void add_sources(octx *c) {
  const double Tn0 = 1000.0, sk1 = 5.0e-5, sk2 = 1.0e-5;
  const double a1_Na = (c->L_ref / c->U_ref) * (c->m_Na / c->rho_ref) * 1e6;
  const double a4 = (c->L_ref / c->U_ref);
  const double a5 = (3.0 * c->L_ref * c->k_Boltz * c->n_ref) / (c->rho_ref * c->U_ref * c->U_ref * c->U_ref);
  const double a6 = (1.0e6 * c->L_ref * c->k_Boltz) / (c->rho_ref * c->U_ref * c->U_ref * c->U_ref * (c->gamma - 1.0));
  for (int i = 0; i < ihi(&c->Jac, 0); ++i)
    for (int j = 0; j < ihi(&c->Jac, 1); ++j)
      for (int k = 0; k < ihi(&c->Jac, 2); ++k) {
        const double upx = V(c->Up, i, j, k, 0), upy = V(c->Up, i, j, k, 1), upz = V(c->Up, i, j, k, 2);
        const double Bx = V(c->Bc, i, j, k, 0), By = V(c->Bc, i, j, k, 1), Bz = V(c->Bc, i, j, k, 2);
        const double Jx = V(c->Jc, i, j, k, 0), Jy = V(c->Jc, i, j, k, 1), Jz = V(c->Jc, i, j, k, 2);
        const double sjbx = Jy * Bz - Jz * By, sjby = Jz * Bx - Jx * Bz, sjbz = Jx * By - Jy * Bx;
        const numinfo num = num_limiter(c, V(c->UH, i, j, k, 0), V(c->UN, i, j, k, 0));
        double dpex = 0.0, dpey = 0.0, dpez = 0.0;
        if (c->ambipolar) {
          const double Vol = fabs(V(c->Jac, i, j, k, 0));
          double ax = 0, ay = 0, az = 0, bx = 0, by = 0, bz = 0, cxm = 0, cym = 0, czm = 0;
          if (Vol > 0.0) {
            ax = 0.5 * (V(c->JDx, i - 1, j, k, 0) + V(c->JDx, i, j, k, 0)) / Vol;
            ay = 0.5 * (V(c->JDx, i - 1, j, k, 1) + V(c->JDx, i, j, k, 1)) / Vol;
            az = 0.5 * (V(c->JDx, i - 1, j, k, 2) + V(c->JDx, i, j, k, 2)) / Vol;
            bx = 0.5 * (V(c->JDy, i, j - 1, k, 0) + V(c->JDy, i, j, k, 0)) / Vol;
            by = 0.5 * (V(c->JDy, i, j - 1, k, 1) + V(c->JDy, i, j, k, 1)) / Vol;
            bz = 0.5 * (V(c->JDy, i, j - 1, k, 2) + V(c->JDy, i, j, k, 2)) / Vol;
            cxm = 0.5 * (V(c->JDz, i, j, k - 1, 0) + V(c->JDz, i, j, k, 0)) / Vol;
            cym = 0.5 * (V(c->JDz, i, j, k - 1, 1) + V(c->JDz, i, j, k, 1)) / Vol;
            czm = 0.5 * (V(c->JDz, i, j, k - 1, 2) + V(c->JDz, i, j, k, 2)) / Vol;
          }
          const double pip = V(c->PVH, i + 1, j, k, 3) + V(c->PVN, i + 1, j, k, 3);
          const double pim = V(c->PVH, i - 1, j, k, 3) + V(c->PVN, i - 1, j, k, 3);
          const double pjp = V(c->PVH, i, j + 1, k, 3) + V(c->PVN, i, j + 1, k, 3);
          const double pjm = V(c->PVH, i, j - 1, k, 3) + V(c->PVN, i, j - 1, k, 3);
          const double pkp = V(c->PVH, i, j, k + 1, 3) + V(c->PVN, i, j, k + 1, 3);
          const double pkm = V(c->PVH, i, j, k - 1, 3) + V(c->PVN, i, j, k - 1, 3);
          dpex = 0.5 * (ax * (pip - pim) + bx * (pjp - pjm) + cxm * (pkp - pkm));
          dpey = 0.5 * (ay * (pip - pim) + by * (pjp - pjm) + cym * (pkp - pkm));
          dpez = 0.5 * (az * (pip - pim) + bz * (pjp - pjm) + czm * (pkp - pkm));
        }
        const double sss = V(c->Photo, i, j, k, 0);
        const double x = V(c->cx, i + 1, j + 1, k + 1, 0), y = V(c->cy, i + 1, j + 1, k + 1, 0), z = V(c->cz, i + 1, j + 1, k + 1, 0);
        const double rho_cyl = sqrt(y * y + z * z);
        const int in_shadow = (x < 0.0 && rho_cyl < 1.0);
        const double vst = in_shadow ? sk2 : sk1;
        for (int s = 0; s < 2; ++s) {
          const ofld *U = s ? &c->UN : &c->UH;
          const ofld *PV = s ? &c->PVN : &c->PVH;
          ofld *R = s ? &c->RN : &c->RH;
          const double nS = s ? num.nNa : num.nH;
          const double chi = s ? num.wNa : num.wH;
          const double rho = dmax(V(*U, i, j, k, 0), 0.0);
          const double u = V(*PV, i, j, k, 0), v = V(*PV, i, j, k, 1), w = V(*PV, i, j, k, 2);
          const double u2 = u * u + v * v + w * w;
          const double subx = (v - upy) * Bz - (w - upz) * By;
          const double suby = (w - upz) * Bx - (u - upx) * Bz;
          const double subz = (u - upx) * By - (v - upy) * Bx;
          const double subu = subx * u + suby * v + subz * w;
          const double sjbu = sjbx * u + sjby * v + sjbz * w;
          const double dpeu = dpex * u + dpey * v + dpez * w;
          const double Ts0 = V(*PV, i, j, k, 4) * c->T_ref;
          double b1, b2;
          if (!s) {
            b1 = vst * (Tn0 - Ts0) * (c->M_H / (c->M_H + c->M_Na));
            b2 = (c->M_Na / (c->M_H + c->M_Na)) * vst;
          } else {
            b1 = vst * (Tn0 - Ts0) * (c->M_Na / (c->M_Na + c->M_Na));
            b2 = (c->M_Na / (c->M_Na + c->M_Na)) * vst;
          }
          V(*R, i, j, k, 1) += c->momentum_induce_coeff * nS * subx + c->momentum_hall_coeff * chi * sjbx;
          V(*R, i, j, k, 2) += c->momentum_induce_coeff * nS * suby + c->momentum_hall_coeff * chi * sjby;
          V(*R, i, j, k, 3) += c->momentum_induce_coeff * nS * subz + c->momentum_hall_coeff * chi * sjbz;
          V(*R, i, j, k, 4) += c->momentum_induce_coeff * nS * subu + c->momentum_hall_coeff * chi * sjbu;
          if (c->ambipolar) {
            V(*R, i, j, k, 1) -= chi * dpex;
            V(*R, i, j, k, 2) -= chi * dpey;
            V(*R, i, j, k, 3) -= chi * dpez;
            V(*R, i, j, k, 4) -= chi * dpeu;
          }
          if (s) {
            V(*R, i, j, k, 0) += a1_Na * sss;
            V(*R, i, j, k, 4) += a6 * sss * Tn0;
          }
          V(*R, i, j, k, 1) -= a4 * rho * u * vst;
          V(*R, i, j, k, 2) -= a4 * rho * v * vst;
          V(*R, i, j, k, 3) -= a4 * rho * w * vst;
          V(*R, i, j, k, 4) -= a4 * rho * u2 * vst;
          V(*R, i, j, k, 4) += a5 * nS * b1;
          V(*R, i, j, k, 4) += a4 * rho * u2 * b2;
        }
      }
}

/* ---- ideal EMF: AssembleOneDirectionEMF_ and AssembleEdgeEMF_FromFaceE_Ideal_
 * (Z4_Mercury/src/physics/MercurySolver_MagExplicit_Ideal.cpp:138-372, 433-594) */
static const ofld *metric_of(const octx *c, int axis) { return axis == 0 ? &c->JDx : axis == 1 ? &c->JDy : &c->JDz; }
static const ofld *bind_of(const octx *c, int axis) { return axis == 0 ? &c->Bx : axis == 1 ? &c->By : &c->Bz; }
static const ofld *badd_of(const octx *c, int axis) { return axis == 0 ? &c->Bax : axis == 1 ? &c->Bay : &c->Baz; }
static inline void shift1(int axis, int *i, int *j, int *k, int s) {
  if (axis == 0) *i += s;
  else if (axis == 1) *j += s;
  else *k += s;
}
static double cell_u_contra(const octx *c, int axis, int i, int j, int k) {
  int ip = i, jp = j, kp = k;
  shift1(axis, &ip, &jp, &kp, 1);
  const ofld *M = metric_of(c, axis);
  const double kx = 0.5 * (*A(M, i, j, k, 0) + *A(M, ip, jp, kp, 0));
  const double ky = 0.5 * (*A(M, i, j, k, 1) + *A(M, ip, jp, kp, 1));
  const double kz = 0.5 * (*A(M, i, j, k, 2) + *A(M, ip, jp, kp, 2));
  const double inv_jac = 1.0 / (fabs(V(c->Jac, i, j, k, 0)) + 1.0e-30);
  return (kx * V(c->Up, i, j, k, 0) + ky * V(c->Up, i, j, k, 1) + kz * V(c->Up, i, j, k, 2)) * inv_jac;
}
static double face_tot(const octx *c, int axis, int i, int j, int k) {
  return *A(bind_of(c, axis), i, j, k, 0) + *A(badd_of(c, axis), i, j, k, 0);
}
static double cell_beta_ind(const octx *c, int axis, int i, int j, int k) {
  int ip = i, jp = j, kp = k;
  shift1(axis, &ip, &jp, &kp, 1);
  return 0.5 * (*A(bind_of(c, axis), i, j, k, 0) + *A(bind_of(c, axis), ip, jp, kp, 0));
}
static double cell_beta_tot(const octx *c, int axis, int i, int j, int k) {
  int ip = i, jp = j, kp = k;
  shift1(axis, &ip, &jp, &kp, 1);
  return 0.5 * (face_tot(c, axis, i, j, k) + face_tot(c, axis, ip, jp, kp));
}
static double emf_flux(const octx *c, int beta_axis, int flux_axis, int iL, int jL, int kL, int iR, int jR, int kR, double bff) {
  const double btL = cell_beta_tot(c, beta_axis, iL, jL, kL), btR = cell_beta_tot(c, beta_axis, iR, jR, kR);
  const double biL = cell_beta_ind(c, beta_axis, iL, jL, kL), biR = cell_beta_ind(c, beta_axis, iR, jR, kR);
  const double ufL = cell_u_contra(c, flux_axis, iL, jL, kL), ufR = cell_u_contra(c, flux_axis, iR, jR, kR);
  const double ubL = cell_u_contra(c, beta_axis, iL, jL, kL), ubR = cell_u_contra(c, beta_axis, iR, jR, kR);
  const double GL = ufL * btL - ubL * bff, GR = ufR * btR - ubR * bff;
  const double r = dmax(fabs(ufL), fabs(ufR));
  return 0.5 * (GL + GR) - 0.5 * r * (biR - biL);
}
static void assemble_face_emf(octx *c, int dir, ofld *EF) {
  const int fa = dir;
  int sub[3] = {0, 0, 0}, sup[3] = {ihi(EF, 0), ihi(EF, 1), ihi(EF, 2)};
  for (int a = 0; a < 3; ++a) {
    sub[a] = (sub[a] - 1 > EF->lo[a] + 1) ? sub[a] - 1 : EF->lo[a] + 1;
    sup[a] = (sup[a] + 1 < EF->hi[a] - 1) ? sup[a] + 1 : EF->hi[a] - 1;
  }
  for (int i = sub[0]; i < sup[0]; ++i)
    for (int j = sub[1]; j < sup[1]; ++j)
      for (int k = sub[2]; k < sup[2]; ++k) {
        int iL = i, jL = j, kL = k;
        shift1(fa, &iL, &jL, &kL, -1);
        const double bff = face_tot(c, fa, i, j, k);
        double e[3] = {0, 0, 0};
        if (fa == 0) {
          const double Ge = emf_flux(c, 1, 0, iL, jL, kL, i, j, k, bff);
          const double Gz = emf_flux(c, 2, 0, iL, jL, kL, i, j, k, bff);
          e[1] = Gz;
          e[2] = -Ge;
        } else if (fa == 1) {
          const double Gx = emf_flux(c, 0, 1, iL, jL, kL, i, j, k, bff);
          const double Gz = emf_flux(c, 2, 1, iL, jL, kL, i, j, k, bff);
          e[0] = -Gz;
          e[2] = Gx;
        } else {
          const double Gx = emf_flux(c, 0, 2, iL, jL, kL, i, j, k, bff);
          const double Ge = emf_flux(c, 1, 2, iL, jL, kL, i, j, k, bff);
          e[0] = Ge;
          e[1] = -Gx;
        }
        V(*EF, i, j, k, 0) = e[0];
        V(*EF, i, j, k, 1) = e[1];
        V(*EF, i, j, k, 2) = e[2];
      }
}
static double max_abs_u4(const octx *c, int axis, int i0, int j0, int k0, int i1, int j1, int k1, int i2, int j2, int k2, int i3,
                         int j3, int k3) {
  double a = 0.0;
  a = dmax(a, fabs(cell_u_contra(c, axis, i0, j0, k0)));
  a = dmax(a, fabs(cell_u_contra(c, axis, i1, j1, k1)));
  a = dmax(a, fabs(cell_u_contra(c, axis, i2, j2, k2)));
  a = dmax(a, fabs(cell_u_contra(c, axis, i3, j3, k3)));
  return a;
}
static void assemble_edge_emf_ideal(octx *c) {
  const double Cuct = 0.5;
  for (int i = 0; i < ihi(&c->Ex, 0); i++)
    for (int j = 0; j < ihi(&c->Ex, 1); j++)
      for (int k = 0; k < ihi(&c->Ex, 2); k++) {
        const double Ec = 0.25 * (V(c->EFy, i, j, k, 0) + V(c->EFy, i, j, k - 1, 0) + V(c->EFz, i, j, k, 0) + V(c->EFz, i, j - 1, k, 0));
        const double ae = max_abs_u4(c, 1, i, j, k, i, j - 1, k, i, j, k - 1, i, j - 1, k - 1);
        const double az = max_abs_u4(c, 2, i, j, k, i, j - 1, k, i, j, k - 1, i, j - 1, k - 1);
        const double d1 = V(c->Bz, i, j, k, 0) - V(c->Bz, i, j - 1, k, 0);
        const double d2 = V(c->By, i, j, k, 0) - V(c->By, i, j, k - 1, 0);
        V(c->Ex, i, j, k, 0) = Ec + Cuct * (0.5 * ae * d1 - 0.5 * az * d2);
      }
  for (int i = 0; i < ihi(&c->Ey, 0); i++)
    for (int j = 0; j < ihi(&c->Ey, 1); j++)
      for (int k = 0; k < ihi(&c->Ey, 2); k++) {
        const double Ec = 0.25 * (V(c->EFx, i, j, k, 1) + V(c->EFx, i, j, k - 1, 1) + V(c->EFz, i, j, k, 1) + V(c->EFz, i - 1, j, k, 1));
        const double az = max_abs_u4(c, 2, i, j, k, i - 1, j, k, i, j, k - 1, i - 1, j, k - 1);
        const double ax = max_abs_u4(c, 0, i, j, k, i - 1, j, k, i, j, k - 1, i - 1, j, k - 1);
        const double d1 = V(c->Bx, i, j, k, 0) - V(c->Bx, i, j, k - 1, 0);
        const double d2 = V(c->Bz, i, j, k, 0) - V(c->Bz, i - 1, j, k, 0);
        V(c->Ey, i, j, k, 0) = Ec + Cuct * (0.5 * az * d1 - 0.5 * ax * d2);
      }
  for (int i = 0; i < ihi(&c->Ez, 0); i++)
    for (int j = 0; j < ihi(&c->Ez, 1); j++)
      for (int k = 0; k < ihi(&c->Ez, 2); k++) {
        const double Ec = 0.25 * (V(c->EFx, i, j, k, 2) + V(c->EFx, i, j - 1, k, 2) + V(c->EFy, i, j, k, 2) + V(c->EFy, i - 1, j, k, 2));
        const double ax = max_abs_u4(c, 0, i, j, k, i - 1, j, k, i, j - 1, k, i - 1, j - 1, k);
        const double ae = max_abs_u4(c, 1, i, j, k, i - 1, j, k, i, j - 1, k, i - 1, j - 1, k);
        const double d1 = V(c->By, i, j, k, 0) - V(c->By, i - 1, j, k, 0);
        const double d2 = V(c->Bx, i, j, k, 0) - V(c->Bx, i, j - 1, k, 0);
        V(c->Ez, i, j, k, 0) = Ec + Cuct * (0.5 * ax * d1 - 0.5 * ae * d2);
      }
}

/* AddAmbipolarEdgeEMF_ (Z4_Mercury/src/physics/MercurySolver_MagExplicit_Ambipo.cpp:3-143) */
static double pe_node(const octx *c, int i, int j, int k) {
  double sum = 0.0;
  for (int di = -1; di <= 0; ++di)
    for (int dj = -1; dj <= 0; ++dj)
      for (int dk = -1; dk <= 0; ++dk) sum += V(c->PVH, i + di, j + dj, k + dk, 3) + V(c->PVN, i + di, j + dj, k + dk, 3);
  return 0.125 * sum;
}
static void add_ambipolar(octx *c) {
  if (!c->ambipolar) return;
  const double pc = (c->rho_ref * c->U_ref) / (c->q_e * c->L_ref * c->B_ref * c->n_ref);
  for (int i = 0; i < ihi(&c->Ex, 0); ++i)
    for (int j = 0; j < ihi(&c->Ex, 1); ++j)
      for (int k = 0; k < ihi(&c->Ex, 2); ++k) {
        const double p0 = pe_node(c, i, j, k), p1 = pe_node(c, i + 1, j, k);
        double rH = 0.0, rN = 0.0;
        for (int dj = -1; dj <= 0; ++dj)
          for (int dk = -1; dk <= 0; ++dk) {
            rH += V(c->UH, i, j + dj, k + dk, 0);
            rN += V(c->UN, i, j + dj, k + dk, 0);
          }
        const numinfo d = num_limiter(c, 0.25 * rH, 0.25 * rN);
        V(c->Ex, i, j, k, 0) -= pc * (p1 - p0) / d.ne_eff;
      }
  for (int i = 0; i < ihi(&c->Ey, 0); ++i)
    for (int j = 0; j < ihi(&c->Ey, 1); ++j)
      for (int k = 0; k < ihi(&c->Ey, 2); ++k) {
        const double p0 = pe_node(c, i, j, k), p1 = pe_node(c, i, j + 1, k);
        double rH = 0.0, rN = 0.0;
        for (int di = -1; di <= 0; ++di)
          for (int dk = -1; dk <= 0; ++dk) {
            rH += V(c->UH, i + di, j, k + dk, 0);
            rN += V(c->UN, i + di, j, k + dk, 0);
          }
        const numinfo d = num_limiter(c, 0.25 * rH, 0.25 * rN);
        V(c->Ey, i, j, k, 0) -= pc * (p1 - p0) / d.ne_eff;
      }
  for (int i = 0; i < ihi(&c->Ez, 0); ++i)
    for (int j = 0; j < ihi(&c->Ez, 1); ++j)
      for (int k = 0; k < ihi(&c->Ez, 2); ++k) {
        const double p0 = pe_node(c, i, j, k), p1 = pe_node(c, i, j, k + 1);
        double rH = 0.0, rN = 0.0;
        for (int di = -1; di <= 0; ++di)
          for (int dj = -1; dj <= 0; ++dj) {
            rH += V(c->UH, i + di, j + dj, k, 0);
            rN += V(c->UN, i + di, j + dj, k, 0);
          }
        const numinfo d = num_limiter(c, 0.25 * rH, 0.25 * rN);
        V(c->Ez, i, j, k, 0) -= pc * (p1 - p0) / d.ne_eff;
      }
}

/* BuildHallFaceEMF_Rusanov_diff_ (Z4_Mercury/src/physics/MercurySolver_MagExplicit_Hall.cpp:58-433);
 * the radial taper per edge (Hall.cpp:6-25) is an input array (tp*). */
static void build_hall(octx *c) {
  const double eps = 1e-14, Cwh = 0.1;
  for (int i = c->Bc.lo[0]; i < c->Bc.hi[0]; ++i)
    for (int j = c->Bc.lo[1]; j < c->Bc.hi[1]; ++j)
      for (int k = c->Bc.lo[2]; k < c->Bc.hi[2]; ++k) {
        const numinfo d = num_limiter(c, V(c->UH, i, j, k, 0), V(c->UN, i, j, k, 0));
        const double alpha = c->hall_coef / d.ne_eff;
        const double Jx = V(c->Jc, i, j, k, 0), Jy = V(c->Jc, i, j, k, 1), Jz = V(c->Jc, i, j, k, 2);
        const double Bx = V(c->Bc, i, j, k, 0), By = V(c->Bc, i, j, k, 1), Bz = V(c->Bc, i, j, k, 2);
        V(c->Ehc, i, j, k, 0) = alpha * (Jy * Bz - Jz * By);
        V(c->Ehc, i, j, k, 1) = alpha * (Jz * Bx - Jx * Bz);
        V(c->Ehc, i, j, k, 2) = alpha * (Jx * By - Jy * Bx);
        V(c->beta, i, j, k, 0) = fabs(alpha) * sqrt(Bx * Bx + By * By + Bz * Bz);
      }
#define AVG4(a, b, cc, d) (0.25 * ((a) + (b) + (cc) + (d)))
  for (int i = 0; i < ihi(&c->Hx, 0); ++i)
    for (int j = 0; j < ihi(&c->Hx, 1); ++j)
      for (int k = 0; k < ihi(&c->Hx, 2); ++k) {
        double Ec[3];
        for (int q = 0; q < 3; ++q)
          Ec[q] = AVG4(V(c->Ehc, i, j - 1, k - 1, q), V(c->Ehc, i, j - 1, k, q), V(c->Ehc, i, j, k - 1, q), V(c->Ehc, i, j, k, q));
        const double Ecen = Ec[0] * V(c->drx, i, j, k, 0) + Ec[1] * V(c->drx, i, j, k, 1) + Ec[2] * V(c->drx, i, j, k, 2);
        const double be = dmax(dmax(V(c->beta, i, j - 1, k - 1, 0), V(c->beta, i, j - 1, k, 0)), dmax(V(c->beta, i, j, k - 1, 0), V(c->beta, i, j, k, 0)));
        const double L = dmax(V(c->dlx, i, j, k, 0), eps);
        const double Abz = 0.5 * (V(c->Az, i, j, k, 0) + V(c->Az, i, j - 1, k, 0));
        const double ihe = L / dmax(Abz, eps);
        const double mue = Cwh * be * ihe * ihe;
        const double Abe = 0.5 * (V(c->Ay, i, j, k, 0) + V(c->Ay, i, j, k - 1, 0));
        const double ihz = L / dmax(Abe, eps);
        const double muz = Cwh * be * ihz * ihz;
        const double d1 = V(c->Bz, i, j, k, 0) - V(c->Bz, i, j - 1, k, 0);
        const double d2 = V(c->By, i, j, k, 0) - V(c->By, i, j, k - 1, 0);
        V(c->Hx, i, j, k, 0) = V(c->tpx, i, j, k, 0) * (Ecen + 0.5 * mue * d1 - 0.5 * muz * d2);
      }
  for (int i = 0; i < ihi(&c->Hy, 0); ++i)
    for (int j = 0; j < ihi(&c->Hy, 1); ++j)
      for (int k = 0; k < ihi(&c->Hy, 2); ++k) {
        double Ec[3];
        for (int q = 0; q < 3; ++q)
          Ec[q] = AVG4(V(c->Ehc, i - 1, j, k - 1, q), V(c->Ehc, i - 1, j, k, q), V(c->Ehc, i, j, k - 1, q), V(c->Ehc, i, j, k, q));
        const double Ecen = Ec[0] * V(c->dry, i, j, k, 0) + Ec[1] * V(c->dry, i, j, k, 1) + Ec[2] * V(c->dry, i, j, k, 2);
        const double be = dmax(dmax(V(c->beta, i - 1, j, k - 1, 0), V(c->beta, i - 1, j, k, 0)), dmax(V(c->beta, i, j, k - 1, 0), V(c->beta, i, j, k, 0)));
        const double L = dmax(V(c->dly, i, j, k, 0), eps);
        const double Abx = 0.5 * (V(c->Ax, i, j, k, 0) + V(c->Ax, i, j, k - 1, 0));
        const double ihz = L / dmax(Abx, eps);
        const double muz = Cwh * be * ihz * ihz;
        const double Abz = 0.5 * (V(c->Az, i, j, k, 0) + V(c->Az, i - 1, j, k, 0));
        const double ihx = L / dmax(Abz, eps);
        const double mux = Cwh * be * ihx * ihx;
        const double d1 = V(c->Bx, i, j, k, 0) - V(c->Bx, i, j, k - 1, 0);
        const double d2 = V(c->Bz, i, j, k, 0) - V(c->Bz, i - 1, j, k, 0);
        V(c->Hy, i, j, k, 0) = V(c->tpy, i, j, k, 0) * (Ecen + 0.5 * muz * d1 - 0.5 * mux * d2);
      }
  for (int i = 0; i < ihi(&c->Hz, 0); ++i)
    for (int j = 0; j < ihi(&c->Hz, 1); ++j)
      for (int k = 0; k < ihi(&c->Hz, 2); ++k) {
        double Ec[3];
        for (int q = 0; q < 3; ++q)
          Ec[q] = AVG4(V(c->Ehc, i - 1, j - 1, k, q), V(c->Ehc, i - 1, j, k, q), V(c->Ehc, i, j - 1, k, q), V(c->Ehc, i, j, k, q));
        const double Ecen = Ec[0] * V(c->drz, i, j, k, 0) + Ec[1] * V(c->drz, i, j, k, 1) + Ec[2] * V(c->drz, i, j, k, 2);
        const double be = dmax(dmax(V(c->beta, i - 1, j - 1, k, 0), V(c->beta, i - 1, j, k, 0)), dmax(V(c->beta, i, j - 1, k, 0), V(c->beta, i, j, k, 0)));
        const double L = dmax(V(c->dlz, i, j, k, 0), eps);
        const double Abe = 0.5 * (V(c->Ay, i, j, k, 0) + V(c->Ay, i - 1, j, k, 0));
        const double ihx = L / dmax(Abe, eps);
        const double mux = Cwh * be * ihx * ihx;
        const double Abx = 0.5 * (V(c->Ax, i, j, k, 0) + V(c->Ax, i, j - 1, k, 0));
        const double ihe = L / dmax(Abx, eps);
        const double mue = Cwh * be * ihe * ihe;
        const double d1 = V(c->By, i, j, k, 0) - V(c->By, i - 1, j, k, 0);
        const double d2 = V(c->Bx, i, j, k, 0) - V(c->Bx, i, j - 1, k, 0);
        V(c->Hz, i, j, k, 0) = V(c->tpz, i, j, k, 0) * (Ecen + 0.5 * mux * d1 - 0.5 * mue * d2);
      }
#undef AVG4
}

static void zero_all(ofld *f) {
  const long tot = (long)(f->hi[0] - f->lo[0]) * (f->hi[1] - f->lo[1]) * (f->hi[2] - f->lo[2]) * f->nc;
  memset(f->p, 0, sizeof(double) * tot);
}
static void zero_inner(ofld *f) {
  for (int i = 0; i < ihi(f, 0); ++i)
    for (int j = 0; j < ihi(f, 1); ++j)
      for (int k = 0; k < ihi(f, 2); ++k)
        for (int m = 0; m < f->nc; ++m) *A(f, i, j, k, m) = 0.0;
}

/* AssembleRHS_Induction_CT_ (Z4_Mercury/src/physics/MercurySolver_MagneticRHS.cpp:90-171) */
static void assemble_induction(octx *c) {
  const int n = c->n;
  zero_all(&c->Ex);
  zero_all(&c->Ey);
  zero_all(&c->Ez);
  assemble_face_emf(c, 0, &c->EFx);
  assemble_face_emf(c, 1, &c->EFy);
  assemble_face_emf(c, 2, &c->EFz);
  assemble_edge_emf_ideal(c);
  add_ambipolar(c);
  /* artificial resistivity off (arti_eta_max = 0, local off) */
  alias_reduce_edges(&c->Ex, LOC_EXI, n);
  alias_reduce_edges(&c->Ey, LOC_EET, n);
  alias_reduce_edges(&c->Ez, LOC_EZE, n);
  build_hall(c);
  sync_periodic(&c->Hx, LOC_EXI, 0, n);
  sync_periodic(&c->Hy, LOC_EET, 0, n);
  sync_periodic(&c->Hz, LOC_EZE, 0, n);
  ofld *E[3] = {&c->Ex, &c->Ey, &c->Ez}, *H[3] = {&c->Hx, &c->Hy, &c->Hz};
  for (int a = 0; a < 3; ++a)
    for (int i = 0; i < ihi(E[a], 0); ++i)
      for (int j = 0; j < ihi(E[a], 1); ++j)
        for (int k = 0; k < ihi(E[a], 2); ++k) *A(E[a], i, j, k, 0) += *A(H[a], i, j, k, 0);
  sync_periodic(&c->Ex, LOC_EXI, 0, n);
  sync_periodic(&c->Ey, LOC_EET, 0, n);
  sync_periodic(&c->Ez, LOC_EZE, 0, n);
  /* CurlEdgeToFace with multiplier -1 (CTOperators.cpp:6-56) */
  for (int i = 0; i < ihi(&c->RBx, 0); ++i)
    for (int j = 0; j < ihi(&c->RBx, 1); ++j)
      for (int k = 0; k < ihi(&c->RBx, 2); ++k)
        V(c->RBx, i, j, k, 0) = -1.0 * ((V(c->Ey, i, j, k, 0) - V(c->Ey, i, j, k + 1, 0)) + (V(c->Ez, i, j + 1, k, 0) - V(c->Ez, i, j, k, 0)));
  for (int i = 0; i < ihi(&c->RBy, 0); ++i)
    for (int j = 0; j < ihi(&c->RBy, 1); ++j)
      for (int k = 0; k < ihi(&c->RBy, 2); ++k)
        V(c->RBy, i, j, k, 0) = -1.0 * ((V(c->Ex, i, j, k + 1, 0) - V(c->Ex, i, j, k, 0)) + (V(c->Ez, i, j, k, 0) - V(c->Ez, i + 1, j, k, 0)));
  for (int i = 0; i < ihi(&c->RBz, 0); ++i)
    for (int j = 0; j < ihi(&c->RBz, 1); ++j)
      for (int k = 0; k < ihi(&c->RBz, 2); ++k)
        V(c->RBz, i, j, k, 0) = -1.0 * ((V(c->Ex, i, j, k, 0) - V(c->Ex, i, j + 1, k, 0)) + (V(c->Ey, i + 1, j, k, 0) - V(c->Ey, i, j, k, 0)));
}

/* StepOnce (Z4_Mercury/src/MercurySolver_Driver.cpp:21-61) without the
 * resistive substep (is_Mercury_resistance = 0).  Returns the dt used. */
double oracle_step(octx *c) {
  const int n = c->n;
  c->dt = compute_timestep(c);
  zero_inner(&c->RH);
  zero_inner(&c->RN);
  zero_inner(&c->RBx);
  zero_inner(&c->RBy);
  zero_inner(&c->RBz);
  scheme_u(c);
  add_sources(c);
  assemble_induction(c);
  /* ApplyUpdate_Euler_ (Z4_Mercury/src/physics/MercurySolver_Advance.cpp:73-147) */
  ofld *U[2] = {&c->UH, &c->UN}, *R[2] = {&c->RH, &c->RN};
  for (int s = 0; s < 2; ++s)
    for (int i = 0; i < ihi(U[s], 0); ++i)
      for (int j = 0; j < ihi(U[s], 1); ++j)
        for (int k = 0; k < ihi(U[s], 2); ++k)
          for (int m = 0; m < 5; ++m) *A(U[s], i, j, k, m) += c->dt * *A(R[s], i, j, k, m);
  ofld *B[3] = {&c->Bx, &c->By, &c->Bz}, *RB[3] = {&c->RBx, &c->RBy, &c->RBz};
  for (int a = 0; a < 3; ++a)
    for (int i = 0; i < ihi(B[a], 0); ++i)
      for (int j = 0; j < ihi(B[a], 1); ++j)
        for (int k = 0; k < ihi(B[a], 2); ++k) *A(B[a], i, j, k, 0) += c->dt * *A(RB[a], i, j, k, 0);
  c->time += c->dt;
  c->step += 1;
  sync_periodic(&c->UH, LOC_CELL, 1, n);
  sync_periodic(&c->UN, LOC_CELL, 1, n);
  sync_periodic(&c->Bx, LOC_FXI, 0, n);
  sync_periodic(&c->By, LOC_FET, 0, n);
  sync_periodic(&c->Bz, LOC_FZE, 0, n);
  oracle_update_derived(c);
  return c->dt;
}

/* ----------------------------------------------------------------- ABI for ctypes */
size_t oracle_ctx_size(void) { return sizeof(octx); }
size_t oracle_fld_offset(void) { return offsetof(octx, UH); }
size_t oracle_fld_size(void) { return sizeof(ofld); }
int oracle_nfields(void) { return (int)((offsetof(octx, dt) - offsetof(octx, UH)) / sizeof(ofld)); }
void oracle_sync_cell(octx *c, ofld *f, int corner1d) { sync_periodic(f, LOC_CELL, corner1d, c->n); }
double oracle_compute_timestep(octx *c) { return compute_timestep(c); }

/* Raw normalisation inputs -> derived constants, in the reference's own
 * arithmetic order (calc_physical_constant, Tools.cpp:3-48). */
octx *oracle_create(const double *raw, int n, int ambipolar) {
  octx *c = (octx *)calloc(1, sizeof(octx));
  const double gamma = raw[0], NA = raw[1], R_uni = raw[2], mu0 = raw[3], q_e = raw[4];
  const double U_ref = raw[5], T_ref = raw[6], n_ref = raw[7], M_ref = raw[8], B_ref = raw[9], L_ref = raw[10];
  const double M_H = raw[11], M_Na = raw[12], CFL = raw[13];
  c->gamma = gamma;
  c->q_e = q_e;
  c->k_Boltz = R_uni / NA;
  c->mu0 = mu0;
  c->U_ref = U_ref;
  c->L_ref = L_ref;
  c->B_ref = B_ref;
  c->T_ref = T_ref;
  c->n_ref = n_ref;
  c->M_ref = M_ref;
  c->rho_ref = M_ref * n_ref / NA;
  c->M_H = M_H;
  c->M_Na = M_Na;
  c->m_Na = M_Na / NA;
  c->state_coeff_H = (R_uni * T_ref) / (M_H * U_ref * U_ref);
  c->state_coeff_Na = (R_uni * T_ref) / (M_Na * U_ref * U_ref);
  c->CFL = CFL;
  c->hall_coef = B_ref * M_ref / (U_ref * q_e * L_ref * mu0 * c->rho_ref * NA);
  c->momentum_induce_coeff = (q_e * L_ref * B_ref * n_ref) / (c->rho_ref * U_ref);
  c->momentum_hall_coeff = (B_ref * B_ref) / (mu0 * c->rho_ref * U_ref * U_ref);
  c->inver_MA2 = B_ref * B_ref / (U_ref * U_ref * mu0 * c->rho_ref);
  c->ne_hall_floor = 0.01;
  c->ambipolar = ambipolar;
  c->n = n;
  return c;
}
void oracle_destroy(octx *c) { free(c); }
void oracle_bind(octx *c, int slot, double *p, const int *lo, const int *hi, int nc) {
  ofld *f = &c->UH + slot;
  f->p = p;
  for (int a = 0; a < 3; ++a) {
    f->lo[a] = lo[a];
    f->hi[a] = hi[a];
  }
  f->nc = nc;
}
double oracle_get_dt(const octx *c) { return c->dt; }
double oracle_get_time(const octx *c) { return c->time; }

/* MercuryBoundary::Sync("Ucell") and Sync("Bface") on the periodic block. */
void oracle_sync_state(octx *c) {
  sync_periodic(&c->UH, LOC_CELL, 1, c->n);
  sync_periodic(&c->UN, LOC_CELL, 1, c->n);
  sync_periodic(&c->Bx, LOC_FXI, 0, c->n);
  sync_periodic(&c->By, LOC_FET, 0, c->n);
  sync_periodic(&c->Bz, LOC_FZE, 0, c->n);
}
