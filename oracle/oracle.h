/* CPU oracle: a plain-C restatement of ExaHyPE's generic nonlinear ADER-DG kernels
 * (ExaHyPE/kernels/aderdg/generic/c/{2d,3d}/<kernel>.cpph). TEST INFRASTRUCTURE ONLY: tests, the
 * smoke check and bench.py's CPU-baseline leg call it as the checker; the product never links it.
 *
 * Parity of this restatement is pinned by tests/test_oracle.py against (a) the reference's own
 * known-answer arrays (generic_euler_testdata.cpp, parsed into tests/golden/ fixtures) and (b) the
 * reference's own kernels compiled in place (oracle/_ref) on seeded non-constant cells.
 *
 * Layouts follow the reference exactly (row-major, last index fastest):
 *   luh     [z][y][x][D]            (2D: [y][x][D]),  D = nVar + nPar
 *   lQi     [z][y][x][t][D]
 *   lFi     [t][z][y][x][d+1][nVar] (slot d = source/NCP)
 *   lQhi    [z][y][x][D]
 *   lFhi    d+1 blocks of n^d*nVar: x as [z][y][x], y as [z][x][y], z as [y][x][z], source [z][y][x]
 *   lQhbnd  [2d][a][b][D], lFhbnd [2d][a][b][nVar]; face 2*dir+orientation; (a,b) = the two
 *           tangential coordinates, slower first (x faces (z,y), y faces (z,x), z faces (y,x)).
 */
#ifndef EXA_ORACLE_H
#define EXA_ORACLE_H
#ifdef __cplusplus
extern "C" {
#endif

enum { EXO_PDE_EULER = 0, EXO_PDE_SWE = 1, EXO_PDE_ACOUSTIC = 2, EXO_PDE_ELASTIC = 3 };

typedef struct {
  int dim;      /* 2 or 3 */
  int order;    /* N; n = N+1 nodes per axis */
  int nvar;     /* number of evolved variables */
  int npar;     /* number of material parameters appended to every node */
  int pde;      /* EXO_PDE_* */
  int use_ncp;  /* non-conservative product active (gradients + fluctuation split) */
  double cfl;   /* CFL safety factor (0.9) */
  double pnpm;  /* ADER-DG PNPM factor for this order */
  int max_picard; /* 0: 2(N+1) with the residual test; >0: that fixed count, no test */
  int has_src;    /* point source active (algebraicSource of the acoustic / elastic systems) */
  double src[8];  /* x, y, z, f0, t0, amplitude, width, variable */
} exo_cfg;

/* DG operator tables on [0,1] for order N (arrays of n and n*n doubles, [row][col]). */
int exo_tables(int order, double* nodes, double* weights, double* Kxi, double* iK1, double* dudx,
               double* F0, double* F1);

/* Per-cell kernels (reference semantics). Returns the reference's Picard return value
 * (3D: index of the converged iteration; 2D: MaxIterations+2 when converged, a reference quirk),
 * and the number of Picard sweeps actually executed in *sweeps (may be NULL). */
int exo_predictor(const exo_cfg* c, const double* luh, const double* centre, const double* dx, double t,
                  double dt, double* lQi, double* lFi, double* lQhi, double* lFhi, double* lQhbnd,
                  double* lFhbnd, int* sweeps);
void exo_volume(const exo_cfg* c, double* lduh, const double* lFhi, const double* dx);
void exo_riemann(const exo_cfg* c, double* FL, double* FR, const double* QL, const double* QR,
                 const double* dx, int direction);
void exo_surface(const exo_cfg* c, double* lduh, const double* lFhbnd, const double* dx);
void exo_face(const exo_cfg* c, double* lduh, const double* lFhbnd_face, int direction, int orientation,
              const double* dx);
void exo_update(const exo_cfg* c, double* luh, const double* luhOld, const double* lduh, double dt);
double exo_dt(const exo_cfg* c, const double* luh, const double* dx);
void exo_boundary_wall(const exo_cfg* c, double* FOut, double* QOut, const double* QIn, int normal);
void exo_flux(const exo_cfg* c, const double* Q, double* F /* [d][nvar] */);
void exo_eigenvalues(const exo_cfg* c, const double* Q, int direction, double* lambda);

/* Uniform patch in the global non-fused order (dt from CFL unless fixed_dt > 0). walls selects
 * the domain faces: 0 periodic, 1 reflective walls, 3 outflow (ghost = inner state). luh: all cells, cell-major,
 * c = (iz*ny+iy)*nx+ix. Optional outputs: dts[nsteps], picard[nsteps*ncells] (sweeps). */
int exo_run(const exo_cfg* c, const int* ncell, const double* offset, const double* size, int walls,
            double* luh, int nsteps, double t0, double fixed_dt, double* t_out, double* dts, int* picard,
            int nthreads);

#ifdef __cplusplus
}
#endif
#endif
