/*
 * mt3d_oracle.c -- CPU oracle for the 3D-MT forward/adjoint solve.
 *
 * TEST INFRASTRUCTURE ONLY.  This file restates, in plain C, the algorithm of
 * ModEM's matrix-free (MF) 3D-MT forward solver so that the CUDA product path
 * can be checked against it.  Only tests/, __graft_entry__.smoke() and the
 * cpu_baseline leg of bench.py may load the library built from it; the product
 * never calls it.
 *
 * Parity unpinned against the reference's own outputs: the reference cannot
 * be built here (Fortran, no compiler) and its forward fixture
 * (unit_testing/3D/CylinderModel_1per.dat) needs the 2-D boundary solver and
 * the impedance functional, which this file does not restate.  The tests pin
 * it by a closed-form layered solution, direct solves and operator identities.
 *
 * Every routine cites the reference routine it restates (paths relative to the
 * ModEM-GPU source tree).  Indices in the loops are kept 1-based, as in the
 * Fortran, through the IEX/IEY/IEZ/IND/ICL macros, so that each loop can be
 * compared line by line with the routine it restates.  The arithmetic is kept
 * in the reference's order so that the oracle reproduces the reference to the
 * last bits wherever the reference is deterministic.
 *
 * Layout of an edge vector (reference getCvector order,
 * f90/3D_MT/SP_Topology/vecTranslate.f90:41-79):
 *   [ Ex(nx, ny+1, nz+1) | Ey(nx+1, ny, nz+1) | Ez(nx+1, ny+1, nz) ]
 * each block column-major (x fastest).  Node scalars: (nx+1, ny+1, nz+1).
 * Cells: (nx, ny, nz).
 */
#include <complex.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

typedef double complex cplx;

/* f90/UTILS/math_constants.f90:12-19.  PI carries the reference's typo and
 * SIGMA_AIR is a default-kind (single precision) literal promoted to double. */
#define ORC_PI 3.14159265357898
static const double MU_0 = ORC_PI * 0.0000004;
static const double SIGMA_AIR = (double)1.0e-10f;
#define ISIGN (-1)

enum { ORC_QMR = 0, ORC_BICG = 1, ORC_COCG = 2 };
enum { ORC_PC_DILU = 0, ORC_PC_JACOBI = 1, ORC_PC_RBDILU = 2, ORC_PC_DILU_SWEEP = 3, ORC_PC_ZLINE = 4 };

typedef struct orc {
    int nx, ny, nz, nzAir;
    double *dx, *dy, *dz;       /* 1-based */
    double *delX, *delY, *delZ; /* 1-based, n+1 entries */
    long nXe, nYe, nZe, nE, nN, nC;
    /* curl-curl tables, CurlcurleSetUp (f90/3D_MT/FWD/modelOperator3D.f90:357-497) */
    int ldx, ldy, ldz;
    double *xXY1, *xXY2, *xXZ1, *xXZ2, *xY, *xZ, *xXO;
    double *yYZ1, *yYZ2, *yYX1, *yYX2, *yZ, *yX, *yYO;
    double *zZX1, *zZX2, *zZY1, *zZY2, *zX, *zY, *zZO;
    double *VE, *VN, *VC;
    double *sigE;   /* edge conductivity, air zeroed as DivCorrSetUp leaves it */
    double *sigC;   /* cell conductivity (ModelParamToCell) */
    cplx *Adiag, *Dilu;
    double *db1, *db2, *c, *d;
    double omega;
    /* solver control (emsolve_control, f90/3D_MT/FWD/EMsolve3D.f90:22-68) */
    int IterPerDivCor, MaxDivCor, MaxIterDivCor;
    double tolEMfwd, tolEMadj, tolDivCor;
    int solver, precond;
    int nsweep;      /* Jacobi sweeps per triangular solve (ORC_PC_DILU_SWEEP) */
    cplx *Drb;       /* 1/D of the red-black ordered D-ILU */
    /* diagnostics (emsolve_diag) */
    int nIterTotal, nDivCor, failed;
    double *EMrelErr;     /* MaxDivCor*IterPerDivCor */
    double *divJ;         /* 2*MaxDivCor */
    double *DivCorRelErr; /* MaxIterDivCor*MaxDivCor */
    int *DivCorIters;     /* MaxDivCor */
} orc_t;

#define IEX(o, ix, iy, iz) ((long)((ix)-1) + (long)(o)->nx * ((long)((iy)-1) + (long)((o)->ny + 1) * ((iz)-1)))
#define IEY(o, ix, iy, iz) ((o)->nXe + (long)((ix)-1) + (long)((o)->nx + 1) * ((long)((iy)-1) + (long)(o)->ny * ((iz)-1)))
#define IEZ(o, ix, iy, iz) ((o)->nXe + (o)->nYe + (long)((ix)-1) + (long)((o)->nx + 1) * ((long)((iy)-1) + (long)((o)->ny + 1) * ((iz)-1)))
#define IND(o, ix, iy, iz) ((long)((ix)-1) + (long)((o)->nx + 1) * ((long)((iy)-1) + (long)((o)->ny + 1) * ((iz)-1)))
#define ICL(o, ix, iy, iz) ((long)((ix)-1) + (long)(o)->nx * ((long)((iy)-1) + (long)(o)->ny * ((iz)-1)))
/* 2-D coefficient tables with 1-based indices */
#define TX(t, i, j) (o->t[(i) + (long)o->ldx * (j)])
#define TY(t, i, j) (o->t[(i) + (long)o->ldy * (j)])

static void *xcalloc(size_t n, size_t s)
{
    void *p = calloc(n ? n : 1, s);
    if (!p) { fprintf(stderr, "oracle: out of memory\n"); abort(); }
    return p;
}

/* ------------------------------------------------------------------------ */
/* grid set-up: setup_grid (f90/3D_MT/GridDef.f90:301-399), metric elements  */
/* EdgeVolume/NodeVolume/CellVolume (f90/3D_MT/GridCalc.f90:44-200)          */
/* ------------------------------------------------------------------------ */
static void curlcurl_setup(orc_t *o);
static void rbdilu_setup(orc_t *o, int adjt);

orc_t *orc_create(int nx, int ny, int nz, int nzAir, const double *dx, const double *dy, const double *dz)
{
    orc_t *o = xcalloc(1, sizeof(orc_t));
    o->nx = nx; o->ny = ny; o->nz = nz; o->nzAir = nzAir;
    o->dx = xcalloc(nx + 2, sizeof(double));
    o->dy = xcalloc(ny + 2, sizeof(double));
    o->dz = xcalloc(nz + 2, sizeof(double));
    o->delX = xcalloc(nx + 2, sizeof(double));
    o->delY = xcalloc(ny + 2, sizeof(double));
    o->delZ = xcalloc(nz + 2, sizeof(double));
    for (int i = 1; i <= nx; i++) o->dx[i] = dx[i - 1];
    for (int i = 1; i <= ny; i++) o->dy[i] = dy[i - 1];
    for (int i = 1; i <= nz; i++) o->dz[i] = dz[i - 1];
    /* GridDef.f90: delX(1)=dx(1); delX(i)=dx(i-1)+dx(i); delX(nx+1)=dx(nx); /2 */
    o->delX[1] = o->dx[1];
    for (int i = 2; i <= nx; i++) o->delX[i] = o->dx[i - 1] + o->dx[i];
    o->delX[nx + 1] = o->dx[nx];
    for (int i = 1; i <= nx + 1; i++) o->delX[i] = o->delX[i] / 2.0;
    o->delY[1] = o->dy[1];
    for (int i = 2; i <= ny; i++) o->delY[i] = o->dy[i - 1] + o->dy[i];
    o->delY[ny + 1] = o->dy[ny];
    for (int i = 1; i <= ny + 1; i++) o->delY[i] = o->delY[i] / 2.0;
    o->delZ[1] = o->dz[1];
    for (int i = 2; i <= nz; i++) o->delZ[i] = o->dz[i - 1] + o->dz[i];
    o->delZ[nz + 1] = o->dz[nz];
    for (int i = 1; i <= nz + 1; i++) o->delZ[i] = o->delZ[i] / 2.0;

    o->nXe = (long)nx * (ny + 1) * (nz + 1);
    o->nYe = (long)(nx + 1) * ny * (nz + 1);
    o->nZe = (long)(nx + 1) * (ny + 1) * nz;
    o->nE = o->nXe + o->nYe + o->nZe;
    o->nN = (long)(nx + 1) * (ny + 1) * (nz + 1);
    o->nC = (long)nx * ny * nz;

    /* EdgeVolume = EdgeLength * EdgeArea (GridCalc.f90:44-90, 190-250) */
    o->VE = xcalloc(o->nE, sizeof(double));
    for (int iz = 1; iz <= nz + 1; iz++)
        for (int iy = 1; iy <= ny + 1; iy++)
            for (int ix = 1; ix <= nx; ix++)
                o->VE[IEX(o, ix, iy, iz)] = o->dx[ix] * (o->delY[iy] * o->delZ[iz]);
    for (int iz = 1; iz <= nz + 1; iz++)
        for (int iy = 1; iy <= ny; iy++)
            for (int ix = 1; ix <= nx + 1; ix++)
                o->VE[IEY(o, ix, iy, iz)] = o->dy[iy] * (o->delX[ix] * o->delZ[iz]);
    for (int iz = 1; iz <= nz; iz++)
        for (int iy = 1; iy <= ny + 1; iy++)
            for (int ix = 1; ix <= nx + 1; ix++)
                o->VE[IEZ(o, ix, iy, iz)] = o->dz[iz] * (o->delX[ix] * o->delY[iy]);
    /* NodeVolume (GridCalc.f90:128-150) */
    o->VN = xcalloc(o->nN, sizeof(double));
    for (int iz = 1; iz <= nz + 1; iz++)
        for (int iy = 1; iy <= ny + 1; iy++)
            for (int ix = 1; ix <= nx + 1; ix++)
                o->VN[IND(o, ix, iy, iz)] = o->delX[ix] * o->delY[iy] * o->delZ[iz];
    /* CellVolume (GridCalc.f90:155-180) */
    o->VC = xcalloc(o->nC, sizeof(double));
    for (int iz = 1; iz <= nz; iz++)
        for (int iy = 1; iy <= ny; iy++)
            for (int ix = 1; ix <= nx; ix++)
                o->VC[ICL(o, ix, iy, iz)] = o->dx[ix] * o->dy[iy] * o->dz[iz];

    o->sigE = xcalloc(o->nE, sizeof(double));
    o->sigC = xcalloc(o->nC, sizeof(double));
    o->Adiag = xcalloc(o->nE, sizeof(cplx));
    o->Dilu = xcalloc(o->nE, sizeof(cplx));
    o->db1 = xcalloc(o->nE, sizeof(double));
    o->db2 = xcalloc(o->nE, sizeof(double));
    o->c = xcalloc(o->nN, sizeof(double));
    o->d = xcalloc(o->nN, sizeof(double));

    /* MF defaults (f90/3D_MT/FWD/EMsolve3D.f90:58-68) */
    o->IterPerDivCor = 40;
    o->MaxDivCor = 20;
    o->MaxIterDivCor = 100;
    o->tolEMfwd = 1e-7;
    o->tolEMadj = 1e-7;
    o->tolDivCor = 1e-5;
    o->solver = ORC_QMR;
    o->precond = ORC_PC_DILU;
    o->EMrelErr = xcalloc((size_t)o->MaxDivCor * o->IterPerDivCor, sizeof(double));
    o->divJ = xcalloc(2 * (size_t)o->MaxDivCor, sizeof(double));
    o->DivCorRelErr = xcalloc((size_t)o->MaxIterDivCor * o->MaxDivCor, sizeof(double));
    o->DivCorIters = xcalloc(o->MaxDivCor, sizeof(int));
    curlcurl_setup(o);
    return o;
}

void orc_destroy(orc_t *o)
{
    if (!o) return;
    double *bufs[] = {o->dx, o->dy, o->dz, o->delX, o->delY, o->delZ, o->xXY1, o->xXY2, o->xXZ1, o->xXZ2,
                      o->xY, o->xZ, o->xXO, o->yYZ1, o->yYZ2, o->yYX1, o->yYX2, o->yZ, o->yX, o->yYO,
                      o->zZX1, o->zZX2, o->zZY1, o->zZY2, o->zX, o->zY, o->zZO, o->VE, o->VN, o->VC,
                      o->sigE, o->sigC, o->db1, o->db2, o->c, o->d, o->EMrelErr, o->divJ, o->DivCorRelErr};
    for (size_t i = 0; i < sizeof(bufs) / sizeof(bufs[0]); i++) free(bufs[i]);
    free(o->Adiag); free(o->Dilu); free(o->DivCorIters); free(o->Drb);
    free(o);
}

void orc_set_control(orc_t *o, int IterPerDivCor, int MaxDivCor, int MaxIterDivCor, double tolEMfwd,
                     double tolEMadj, double tolDivCor, int solver, int precond)
{
    o->IterPerDivCor = IterPerDivCor;
    o->MaxDivCor = MaxDivCor;
    o->MaxIterDivCor = MaxIterDivCor;
    o->tolEMfwd = tolEMfwd;
    o->tolEMadj = tolEMadj;
    o->tolDivCor = tolDivCor;
    o->solver = solver;
    o->precond = precond % 16;
    o->nsweep = precond / 16;
    if (o->precond == ORC_PC_RBDILU && o->omega > 0) rbdilu_setup(o, 0);
    free(o->EMrelErr); free(o->divJ); free(o->DivCorRelErr); free(o->DivCorIters);
    o->EMrelErr = xcalloc((size_t)MaxDivCor * IterPerDivCor, sizeof(double));
    o->divJ = xcalloc(2 * (size_t)MaxDivCor, sizeof(double));
    o->DivCorRelErr = xcalloc((size_t)MaxIterDivCor * MaxDivCor, sizeof(double));
    o->DivCorIters = xcalloc(MaxDivCor, sizeof(int));
}

/* CurlcurleSetUp, f90/3D_MT/FWD/modelOperator3D.f90:357-497 */
static void curlcurl_setup(orc_t *o)
{
    int nx = o->nx, ny = o->ny, nz = o->nz;
    o->ldx = nx + 2; o->ldy = ny + 2; o->ldz = nz + 2;
    o->xXY1 = xcalloc(o->ldy, sizeof(double)); o->xXY2 = xcalloc(o->ldy, sizeof(double));
    o->xXZ1 = xcalloc(o->ldz, sizeof(double)); o->xXZ2 = xcalloc(o->ldz, sizeof(double));
    o->yYZ1 = xcalloc(o->ldz, sizeof(double)); o->yYZ2 = xcalloc(o->ldz, sizeof(double));
    o->yYX1 = xcalloc(o->ldx, sizeof(double)); o->yYX2 = xcalloc(o->ldx, sizeof(double));
    o->zZX1 = xcalloc(o->ldx, sizeof(double)); o->zZX2 = xcalloc(o->ldx, sizeof(double));
    o->zZY1 = xcalloc(o->ldy, sizeof(double)); o->zZY2 = xcalloc(o->ldy, sizeof(double));
    o->xY = xcalloc((size_t)o->ldx * o->ldy, sizeof(double));
    o->xZ = xcalloc((size_t)o->ldx * o->ldz, sizeof(double));
    o->xXO = xcalloc((size_t)o->ldy * o->ldz, sizeof(double));
    o->yZ = xcalloc((size_t)o->ldy * o->ldz, sizeof(double));
    o->yX = xcalloc((size_t)o->ldx * o->ldy, sizeof(double));
    o->yYO = xcalloc((size_t)o->ldx * o->ldz, sizeof(double));
    o->zX = xcalloc((size_t)o->ldx * o->ldz, sizeof(double));
    o->zY = xcalloc((size_t)o->ldy * o->ldz, sizeof(double));
    o->zZO = xcalloc((size_t)o->ldx * o->ldy, sizeof(double));
    double *dx = o->dx, *dy = o->dy, *dz = o->dz, *delX = o->delX, *delY = o->delY, *delZ = o->delZ;

    for (int iy = 2; iy <= ny; iy++) {
        o->xXY2[iy] = -1.0 / (delY[iy] * dy[iy]);
        o->xXY1[iy] = -1.0 / (delY[iy] * dy[iy - 1]);
    }
    for (int iz = 2; iz <= nz; iz++) {
        o->xXZ2[iz] = -1.0 / (delZ[iz] * dz[iz]);
        o->xXZ1[iz] = -1.0 / (delZ[iz] * dz[iz - 1]);
    }
    for (int iy = 2; iy <= ny; iy++)
        for (int iz = 2; iz <= nz; iz++)
            TY(xXO, iy, iz) = -(o->xXY1[iy] + o->xXY2[iy] + o->xXZ1[iz] + o->xXZ2[iz]);
    for (int ix = 1; ix <= nx; ix++)
        for (int iy = 2; iy <= ny; iy++) TX(xY, ix, iy) = 1.0 / (delY[iy] * dx[ix]);
    for (int ix = 1; ix <= nx; ix++)
        for (int iz = 2; iz <= nz; iz++) TX(xZ, ix, iz) = 1.0 / (delZ[iz] * dx[ix]);

    for (int iz = 2; iz <= nz; iz++) {
        o->yYZ2[iz] = -1.0 / (delZ[iz] * dz[iz]);
        o->yYZ1[iz] = -1.0 / (delZ[iz] * dz[iz - 1]);
    }
    for (int ix = 2; ix <= nx; ix++) {
        o->yYX2[ix] = -1.0 / (delX[ix] * dx[ix]);
        o->yYX1[ix] = -1.0 / (delX[ix] * dx[ix - 1]);
    }
    for (int ix = 2; ix <= nx; ix++)
        for (int iz = 2; iz <= nz; iz++)
            TX(yYO, ix, iz) = -(o->yYX1[ix] + o->yYX2[ix] + o->yYZ1[iz] + o->yYZ2[iz]);
    for (int iy = 1; iy <= ny; iy++)
        for (int iz = 2; iz <= nz; iz++) TY(yZ, iy, iz) = 1.0 / (delZ[iz] * dy[iy]);
    for (int ix = 2; ix <= nx; ix++)
        for (int iy = 1; iy <= ny; iy++) TX(yX, ix, iy) = 1.0 / (delX[ix] * dy[iy]);

    for (int ix = 2; ix <= nx; ix++) {
        o->zZX2[ix] = -1.0 / (delX[ix] * dx[ix]);
        o->zZX1[ix] = -1.0 / (delX[ix] * dx[ix - 1]);
    }
    for (int iy = 2; iy <= ny; iy++) {
        o->zZY2[iy] = -1.0 / (delY[iy] * dy[iy]);
        o->zZY1[iy] = -1.0 / (delY[iy] * dy[iy - 1]);
    }
    for (int ix = 2; ix <= nx; ix++)
        for (int iy = 2; iy <= ny; iy++)
            TX(zZO, ix, iy) = -(o->zZX1[ix] + o->zZX2[ix] + o->zZY1[iy] + o->zZY2[iy]);
    for (int ix = 2; ix <= nx; ix++)
        for (int iz = 1; iz <= nz; iz++) TX(zX, ix, iz) = 1.0 / (delX[ix] * dz[iz]);
    for (int iy = 2; iy <= ny; iy++)
        for (int iz = 1; iz <= nz; iz++) TY(zY, iy, iz) = 1.0 / (delY[iy] * dz[iz]);
}

/* ------------------------------------------------------------------------ */
/* conductivity mapping                                                      */
/* ------------------------------------------------------------------------ */

/* Cell2Edge, f90/3D_MT/GridCalc.f90:430-560 (Cartesian branch) */
static void cell2edge(const orc_t *o, const double *C, double *E)
{
    int nx = o->nx, ny = o->ny, nz = o->nz;
#define CV(ix, iy, iz) C[ICL(o, ix, iy, iz)]
    memset(E, 0, sizeof(double) * o->nE);
    for (int ix = 1; ix <= nx; ix++)
        for (int iy = 2; iy <= ny; iy++)
            for (int iz = 2; iz <= nz; iz++)
                E[IEX(o, ix, iy, iz)] = (CV(ix, iy - 1, iz - 1) + CV(ix, iy, iz - 1) + CV(ix, iy - 1, iz) + CV(ix, iy, iz)) / 4.0;
    for (int ix = 2; ix <= nx; ix++)
        for (int iy = 1; iy <= ny; iy++)
            for (int iz = 2; iz <= nz; iz++)
                E[IEY(o, ix, iy, iz)] = (CV(ix - 1, iy, iz - 1) + CV(ix, iy, iz - 1) + CV(ix - 1, iy, iz) + CV(ix, iy, iz)) / 4.0;
    for (int ix = 2; ix <= nx; ix++)
        for (int iy = 2; iy <= ny; iy++)
            for (int iz = 1; iz <= nz; iz++)
                E[IEZ(o, ix, iy, iz)] = (CV(ix - 1, iy - 1, iz) + CV(ix - 1, iy, iz) + CV(ix, iy - 1, iz) + CV(ix, iy, iz)) / 4.0;
    int iz = 1;
    for (int iy = 1; iy <= ny; iy++)
        for (int ix = 2; ix <= nx; ix++) E[IEY(o, ix, iy, iz)] = (CV(ix - 1, iy, iz) + CV(ix, iy, iz)) / 2.0;
    for (int ix = 1; ix <= nx; ix++)
        for (int iy = 2; iy <= ny; iy++) E[IEX(o, ix, iy, iz)] = (CV(ix, iy - 1, iz) + CV(ix, iy, iz)) / 2.0;
    iz = nz + 1;
    for (int iy = 1; iy <= ny; iy++)
        for (int ix = 2; ix <= nx; ix++) E[IEY(o, ix, iy, iz)] = (CV(ix - 1, iy, iz - 1) + CV(ix, iy, iz - 1)) / 2.0;
    for (int ix = 1; ix <= nx; ix++)
        for (int iy = 2; iy <= ny; iy++) E[IEX(o, ix, iy, iz)] = (CV(ix, iy - 1, iz - 1) + CV(ix, iy, iz - 1)) / 2.0;
    int ix = 1;
    for (int iy = 1; iy <= ny; iy++)
        for (int jz = 2; jz <= nz; jz++) E[IEY(o, ix, iy, jz)] = (CV(ix, iy, jz - 1) + CV(ix, iy, jz)) / 2.0;
    for (int jz = 1; jz <= nz; jz++)
        for (int iy = 2; iy <= ny; iy++) E[IEZ(o, ix, iy, jz)] = (CV(ix, iy - 1, jz) + CV(ix, iy, jz)) / 2.0;
    ix = nx + 1;
    for (int iy = 1; iy <= ny; iy++)
        for (int jz = 2; jz <= nz; jz++) E[IEY(o, ix, iy, jz)] = (CV(ix - 1, iy, jz - 1) + CV(ix - 1, iy, jz)) / 2.0;
    for (int jz = 1; jz <= nz; jz++)
        for (int iy = 2; iy <= ny; iy++) E[IEZ(o, ix, iy, jz)] = (CV(ix - 1, iy - 1, jz) + CV(ix - 1, iy, jz)) / 2.0;
    int iy = 1;
    for (int jx = 1; jx <= nx; jx++)
        for (int jz = 2; jz <= nz; jz++) E[IEX(o, jx, iy, jz)] = (CV(jx, iy, jz - 1) + CV(jx, iy, jz)) / 2.0;
    for (int jz = 1; jz <= nz; jz++)
        for (int jx = 2; jx <= nx; jx++) E[IEZ(o, jx, iy, jz)] = (CV(jx - 1, iy, jz) + CV(jx, iy, jz)) / 2.0;
    iy = ny + 1;
    for (int jx = 1; jx <= nx; jx++)
        for (int jz = 2; jz <= nz; jz++) E[IEX(o, jx, iy, jz)] = (CV(jx, iy - 1, jz - 1) + CV(jx, iy - 1, jz)) / 2.0;
    for (int jz = 1; jz <= nz; jz++)
        for (int jx = 2; jx <= nx; jx++) E[IEZ(o, jx, iy, jz)] = (CV(jx - 1, iy - 1, jz) + CV(jx, iy - 1, jz)) / 2.0;
    for (int jz = 1; jz <= nz; jz++) {
        E[IEZ(o, 1, 1, jz)] = CV(1, 1, jz);
        E[IEZ(o, 1, ny + 1, jz)] = CV(1, ny, jz);
        E[IEZ(o, nx + 1, 1, jz)] = CV(nx, 1, jz);
        E[IEZ(o, nx + 1, ny + 1, jz)] = CV(nx, ny, jz);
    }
    for (int jy = 1; jy <= ny; jy++) {
        E[IEY(o, 1, jy, 1)] = CV(1, jy, 1);
        E[IEY(o, 1, jy, nz + 1)] = CV(1, jy, nz);
        E[IEY(o, nx + 1, jy, 1)] = CV(nx, jy, 1);
        E[IEY(o, nx + 1, jy, nz + 1)] = CV(nx, jy, nz);
    }
    for (int jx = 1; jx <= nx; jx++) {
        E[IEX(o, jx, 1, 1)] = CV(jx, 1, 1);
        E[IEX(o, jx, 1, nz + 1)] = CV(jx, 1, nz);
        E[IEX(o, jx, ny + 1, 1)] = CV(jx, ny, 1);
        E[IEX(o, jx, ny + 1, nz + 1)] = CV(jx, ny, nz);
    }
#undef CV
}

/* Edge2Cell, f90/3D_MT/GridCalc.f90:1047-1226: the transpose of Cell2Edge */
static void edge2cell(const orc_t *o, const double *E, double *C)
{
    int nx = o->nx, ny = o->ny, nz = o->nz;
#define CA(ix, iy, iz, val) (C[ICL(o, ix, iy, iz)] += (val))
    memset(C, 0, sizeof(double) * o->nC);
    for (int ix = 1; ix <= nx; ix++)
        for (int iy = 2; iy <= ny; iy++)
            for (int iz = 2; iz <= nz; iz++) {
                double e = E[IEX(o, ix, iy, iz)];
                CA(ix, iy - 1, iz - 1, e / 4.0); CA(ix, iy, iz - 1, e / 4.0);
                CA(ix, iy - 1, iz, e / 4.0); CA(ix, iy, iz, e / 4.0);
            }
    for (int ix = 2; ix <= nx; ix++)
        for (int iy = 1; iy <= ny; iy++)
            for (int iz = 2; iz <= nz; iz++) {
                double e = E[IEY(o, ix, iy, iz)];
                CA(ix - 1, iy, iz - 1, e / 4.0); CA(ix, iy, iz - 1, e / 4.0);
                CA(ix - 1, iy, iz, e / 4.0); CA(ix, iy, iz, e / 4.0);
            }
    for (int ix = 2; ix <= nx; ix++)
        for (int iy = 2; iy <= ny; iy++)
            for (int iz = 1; iz <= nz; iz++) {
                double e = E[IEZ(o, ix, iy, iz)];
                CA(ix - 1, iy - 1, iz, e / 4.0); CA(ix - 1, iy, iz, e / 4.0);
                CA(ix, iy - 1, iz, e / 4.0); CA(ix, iy, iz, e / 4.0);
            }
    int iz = 1;
    for (int iy = 1; iy <= ny; iy++)
        for (int ix = 2; ix <= nx; ix++) {
            double e = E[IEY(o, ix, iy, iz)];
            CA(ix - 1, iy, iz, e / 2.0); CA(ix, iy, iz, e / 2.0);
        }
    for (int ix = 1; ix <= nx; ix++)
        for (int iy = 2; iy <= ny; iy++) {
            double e = E[IEX(o, ix, iy, iz)];
            CA(ix, iy - 1, iz, e / 2.0); CA(ix, iy, iz, e / 2.0);
        }
    iz = nz + 1;
    for (int iy = 1; iy <= ny; iy++)
        for (int ix = 2; ix <= nx; ix++) {
            double e = E[IEY(o, ix, iy, iz)];
            CA(ix - 1, iy, iz - 1, e / 2.0); CA(ix, iy, iz - 1, e / 2.0);
        }
    for (int ix = 1; ix <= nx; ix++)
        for (int iy = 2; iy <= ny; iy++) {
            double e = E[IEX(o, ix, iy, iz)];
            CA(ix, iy - 1, iz - 1, e / 2.0); CA(ix, iy, iz - 1, e / 2.0);
        }
    int ix = 1;
    for (int iy = 1; iy <= ny; iy++)
        for (int jz = 2; jz <= nz; jz++) {
            double e = E[IEY(o, ix, iy, jz)];
            CA(ix, iy, jz - 1, e / 2.0); CA(ix, iy, jz, e / 2.0);
        }
    for (int jz = 1; jz <= nz; jz++)
        for (int iy = 2; iy <= ny; iy++) {
            double e = E[IEZ(o, ix, iy, jz)];
            CA(ix, iy - 1, jz, e / 2.0); CA(ix, iy, jz, e / 2.0);
        }
    ix = nx + 1;
    for (int iy = 1; iy <= ny; iy++)
        for (int jz = 2; jz <= nz; jz++) {
            double e = E[IEY(o, ix, iy, jz)];
            CA(ix - 1, iy, jz - 1, e / 2.0); CA(ix - 1, iy, jz, e / 2.0);
        }
    for (int jz = 1; jz <= nz; jz++)
        for (int iy = 2; iy <= ny; iy++) {
            double e = E[IEZ(o, ix, iy, jz)];
            CA(ix - 1, iy - 1, jz, e / 2.0); CA(ix - 1, iy, jz, e / 2.0);
        }
    int iy = 1;
    for (int jx = 1; jx <= nx; jx++)
        for (int jz = 2; jz <= nz; jz++) {
            double e = E[IEX(o, jx, iy, jz)];
            CA(jx, iy, jz - 1, e / 2.0); CA(jx, iy, jz, e / 2.0);
        }
    for (int jz = 1; jz <= nz; jz++)
        for (int jx = 2; jx <= nx; jx++) {
            double e = E[IEZ(o, jx, iy, jz)];
            CA(jx - 1, iy, jz, e / 2.0); CA(jx, iy, jz, e / 2.0);
        }
    iy = ny + 1;
    for (int jx = 1; jx <= nx; jx++)
        for (int jz = 2; jz <= nz; jz++) {
            double e = E[IEX(o, jx, iy, jz)];
            CA(jx, iy - 1, jz - 1, e / 2.0); CA(jx, iy - 1, jz, e / 2.0);
        }
    for (int jz = 1; jz <= nz; jz++)
        for (int jx = 2; jx <= nx; jx++) {
            double e = E[IEZ(o, jx, iy, jz)];
            CA(jx - 1, iy - 1, jz, e / 2.0); CA(jx, iy - 1, jz, e / 2.0);
        }
    for (int jz = 1; jz <= nz; jz++) {
        CA(1, 1, jz, E[IEZ(o, 1, 1, jz)]);
        CA(1, ny, jz, E[IEZ(o, 1, ny + 1, jz)]);
        CA(nx, 1, jz, E[IEZ(o, nx + 1, 1, jz)]);
        CA(nx, ny, jz, E[IEZ(o, nx + 1, ny + 1, jz)]);
    }
    for (int jy = 1; jy <= ny; jy++) {
        CA(1, jy, 1, E[IEY(o, 1, jy, 1)]);
        CA(1, jy, nz, E[IEY(o, 1, jy, nz + 1)]);
        CA(nx, jy, 1, E[IEY(o, nx + 1, jy, 1)]);
        CA(nx, jy, nz, E[IEY(o, nx + 1, jy, nz + 1)]);
    }
    for (int jx = 1; jx <= nx; jx++) {
        CA(jx, 1, 1, E[IEX(o, jx, 1, 1)]);
        CA(jx, 1, nz, E[IEX(o, jx, 1, nz + 1)]);
        CA(jx, ny, 1, E[IEX(o, jx, ny + 1, 1)]);
        CA(jx, ny, nz, E[IEX(o, jx, ny + 1, nz + 1)]);
    }
#undef CA
}

/* ModelParamToEdge, LOGE branch (f90/3D_MT/modelParam/ModelMap.inc:88-188).
 * m_earth holds ln(sigma) for the nx*ny*nzEarth earth cells (x fastest). When
 * m0_earth is given, the linearised mapping is used (air set to zero). */
static void model_to_edge(const orc_t *o, const double *m_earth, double airCond, const double *m0_earth,
                          double *Econd)
{
    long nC = o->nC;
    double *temp = xcalloc(nC, sizeof(double));
    double *Ctemp = xcalloc(nC, sizeof(double));
    double *Etemp = xcalloc(o->nE, sizeof(double));
    double *VEg = xcalloc(o->nE, sizeof(double));
    int nzAir = o->nzAir;
    for (int iz = 1; iz <= o->nz; iz++)
        for (int iy = 1; iy <= o->ny; iy++)
            for (int ix = 1; ix <= o->nx; ix++) {
                long ic = ICL(o, ix, iy, iz);
                if (iz <= nzAir) {
                    temp[ic] = m0_earth ? 0.0 : exp(airCond);
                } else {
                    long ie = ic - (long)o->nx * o->ny * nzAir;
                    temp[ic] = m0_earth ? m_earth[ie] * exp(m0_earth[ie]) : exp(m_earth[ie]);
                }
            }
    cell2edge(o, o->VC, VEg);
    for (long i = 0; i < nC; i++) Ctemp[i] = o->VC[i] * temp[i];
    cell2edge(o, Ctemp, Etemp);
    for (long i = 0; i < o->nE; i++) Econd[i] = Etemp[i] / VEg[i];
    free(temp); free(Ctemp); free(Etemp); free(VEg);
}

void orc_model_to_edge(const orc_t *o, const double *m_earth, double airCond, const double *m0_earth,
                       double *Econd)
{
    model_to_edge(o, m_earth, airCond, m0_earth, Econd);
}

/* DivCorrSetUp, f90/3D_MT/FWD/modelOperator3D.f90:1538-1672 */
static void divcorr_setup(orc_t *o)
{
    int nx = o->nx, ny = o->ny, nz = o->nz, nzAir = o->nzAir;
    double *s = o->sigE;
    for (int iz = 1; iz <= nzAir; iz++)
        for (int iy = 1; iy <= ny; iy++)
            for (int ix = 1; ix <= nx; ix++) {
                s[IEX(o, ix, iy, iz)] = SIGMA_AIR;
                s[IEY(o, ix, iy, iz)] = SIGMA_AIR;
                s[IEZ(o, ix, iy, iz)] = SIGMA_AIR;
            }
    memset(o->db1, 0, sizeof(double) * o->nE);
    memset(o->db2, 0, sizeof(double) * o->nE);
    memset(o->c, 0, sizeof(double) * o->nN);
    for (int iz = 2; iz <= nz; iz++)
        for (int iy = 2; iy <= ny; iy++)
            for (int ix = 2; ix <= nx; ix++) {
                long ex = IEX(o, ix, iy, iz), ey = IEY(o, ix, iy, iz), ez = IEZ(o, ix, iy, iz);
                o->db1[ex] = s[IEX(o, ix - 1, iy, iz)] / (o->dx[ix - 1] * o->delX[ix]);
                o->db2[ex] = s[IEX(o, ix, iy, iz)] / (o->dx[ix] * o->delX[ix]);
                o->db1[ey] = s[IEY(o, ix, iy - 1, iz)] / (o->dy[iy - 1] * o->delY[iy]);
                o->db2[ey] = s[IEY(o, ix, iy, iz)] / (o->dy[iy] * o->delY[iy]);
                o->db1[ez] = s[IEZ(o, ix, iy, iz - 1)] / (o->dz[iz - 1] * o->delZ[iz]);
                o->db2[ez] = s[IEZ(o, ix, iy, iz)] / (o->dz[iz] * o->delZ[iz]);
                o->c[IND(o, ix, iy, iz)] = -(o->db1[ex] + o->db2[ex] + o->db1[ey] + o->db2[ey] + o->db1[ez] + o->db2[ez]);
            }
    for (int iz = 1; iz <= nzAir; iz++)
        for (int iy = 1; iy <= ny; iy++)
            for (int ix = 1; ix <= nx; ix++) {
                s[IEX(o, ix, iy, iz)] = 0.0;
                s[IEY(o, ix, iy, iz)] = 0.0;
                s[IEZ(o, ix, iy, iz)] = 0.0;
            }
    for (int iz = 2; iz <= nz; iz++)
        for (int iy = 2; iy <= ny; iy++)
            for (int ix = 2; ix <= nx; ix++) {
                double v = o->VN[IND(o, ix, iy, iz)];
                long ex = IEX(o, ix, iy, iz), ey = IEY(o, ix, iy, iz), ez = IEZ(o, ix, iy, iz);
                o->db1[ex] *= v; o->db1[ey] *= v; o->db1[ez] *= v;
                o->db2[ex] *= v; o->db2[ey] *= v; o->db2[ez] *= v;
            }
    for (long i = 0; i < o->nN; i++) o->c[i] = o->c[i] * o->VN[i];
    /* force coefficients that multiply boundary nodes to zero */
    for (int iz = 1; iz <= nz + 1; iz++)
        for (int iy = 1; iy <= ny + 1; iy++) {
            o->db1[IEX(o, 2, iy, iz)] = 0.0;
            o->db2[IEX(o, nx, iy, iz)] = 0.0;
        }
    for (int iz = 1; iz <= nz + 1; iz++)
        for (int ix = 1; ix <= nx + 1; ix++) {
            o->db1[IEY(o, ix, 2, iz)] = 0.0;
            o->db2[IEY(o, ix, ny, iz)] = 0.0;
        }
    for (int iy = 1; iy <= ny + 1; iy++)
        for (int ix = 1; ix <= nx + 1; ix++) {
            o->db1[IEZ(o, ix, iy, 2)] = 0.0;
            o->db2[IEZ(o, ix, iy, nz)] = 0.0;
        }
    for (int iz = 1; iz <= nz + 1; iz++)
        for (int iy = 1; iy <= ny + 1; iy++)
            for (int ix = 1; ix <= nx + 1; ix++)
                if (ix == 1 || iy == 1 || iz == 1) o->d[IND(o, ix, iy, iz)] = 1.0;
    for (int iz = 2; iz <= nz; iz++)
        for (int iy = 2; iy <= ny; iy++)
            for (int ix = 2; ix <= nx; ix++) {
                long n = IND(o, ix, iy, iz);
                double v = o->c[n]
                    - o->db1[IEX(o, ix, iy, iz)] * o->db2[IEX(o, ix - 1, iy, iz)] * o->d[IND(o, ix - 1, iy, iz)]
                    - o->db1[IEY(o, ix, iy, iz)] * o->db2[IEY(o, ix, iy - 1, iz)] * o->d[IND(o, ix, iy - 1, iz)]
                    - o->db1[IEZ(o, ix, iy, iz)] * o->db2[IEZ(o, ix, iy, iz - 1)] * o->d[IND(o, ix, iy, iz - 1)];
                o->d[n] = 1.0 / v;
            }
}

/* UpdateCond (f90/3D_MT/FWD/modelOperator3D.f90:211-232): ModelParamToEdge,
 * DivCorrSetUp and ModelParamToCell. */
void orc_update_cond(orc_t *o, const double *m_earth, double airCond)
{
    model_to_edge(o, m_earth, airCond, NULL, o->sigE);
    divcorr_setup(o);
    /* ModelParamToCell (ModelMap.inc:26-66) */
    for (int iz = 1; iz <= o->nz; iz++)
        for (int iy = 1; iy <= o->ny; iy++)
            for (int ix = 1; ix <= o->nx; ix++) {
                long ic = ICL(o, ix, iy, iz);
                o->sigC[ic] = (iz <= o->nzAir) ? exp(airCond) : exp(m_earth[ic - (long)o->nx * o->ny * o->nzAir]);
            }
}

/* UpdateFreq: AdiagSetUp + DiluSetUp (f90/3D_MT/FWD/modelOperator3D.f90:196-204, 649-672, 1090-1163) */
void orc_update_freq(orc_t *o, double omega)
{
    int nx = o->nx, ny = o->ny, nz = o->nz;
    o->omega = omega;
    for (long i = 0; i < o->nE; i++) o->Adiag[i] = CMPLX(0.0, 1.0) * omega * MU_0 * o->sigE[i];
    cplx *D = o->Dilu;
    for (long i = 0; i < o->nE; i++) D[i] = 0.0;
    for (int iz = 1; iz <= nz + 1; iz++)
        for (int ix = 1; ix <= nx; ix++) { D[IEX(o, ix, 1, iz)] = 1.0; }
    for (int iy = 1; iy <= ny + 1; iy++)
        for (int ix = 1; ix <= nx; ix++) { D[IEX(o, ix, iy, 1)] = 1.0; }
    for (int iz = 1; iz <= nz + 1; iz++)
        for (int iy = 1; iy <= ny; iy++) { D[IEY(o, 1, iy, iz)] = 1.0; }
    for (int iy = 1; iy <= ny; iy++)
        for (int ix = 1; ix <= nx + 1; ix++) { D[IEY(o, ix, iy, 1)] = 1.0; }
    for (int iz = 1; iz <= nz; iz++)
        for (int iy = 1; iy <= ny + 1; iy++) { D[IEZ(o, 1, iy, iz)] = 1.0; }
    for (int iz = 1; iz <= nz; iz++)
        for (int ix = 1; ix <= nx + 1; ix++) { D[IEZ(o, ix, 1, iz)] = 1.0; }
    for (int ix = 1; ix <= nx; ix++)
        for (int iy = 2; iy <= ny; iy++)
            for (int iz = 2; iz <= nz; iz++) {
                long e = IEX(o, ix, iy, iz);
                cplx v = TY(xXO, iy, iz) - CMPLX(0.0, 1.0) * omega * MU_0 * o->sigE[e]
                         - o->xXY1[iy] * o->xXY2[iy - 1] * D[IEX(o, ix, iy - 1, iz)]
                         - o->xXZ1[iz] * o->xXZ2[iz - 1] * D[IEX(o, ix, iy, iz - 1)];
                D[e] = 1.0 / v;
            }
    for (int iy = 1; iy <= ny; iy++)
        for (int iz = 2; iz <= nz; iz++)
            for (int ix = 2; ix <= nx; ix++) {
                long e = IEY(o, ix, iy, iz);
                cplx v = TX(yYO, ix, iz) - CMPLX(0.0, 1.0) * omega * MU_0 * o->sigE[e]
                         - o->yYZ1[iz] * o->yYZ2[iz - 1] * D[IEY(o, ix, iy, iz - 1)]
                         - o->yYX1[ix] * o->yYX2[ix - 1] * D[IEY(o, ix - 1, iy, iz)];
                D[e] = 1.0 / v;
            }
    for (int iz = 1; iz <= nz; iz++)
        for (int ix = 2; ix <= nx; ix++)
            for (int iy = 2; iy <= ny; iy++) {
                long e = IEZ(o, ix, iy, iz);
                cplx v = TX(zZO, ix, iy) - CMPLX(0.0, 1.0) * omega * MU_0 * o->sigE[e]
                         - o->zZX1[ix] * o->zZX2[ix - 1] * D[IEZ(o, ix - 1, iy, iz)]
                         - o->zZY1[iy] * o->zZY2[iy - 1] * D[IEZ(o, ix, iy - 1, iz)];
                D[e] = 1.0 / v;
            }
    if (o->precond == ORC_PC_RBDILU) rbdilu_setup(o, 0);
}

/* ------------------------------------------------------------------------ */
/* operators                                                                 */
/* ------------------------------------------------------------------------ */

/* Maxwell (f90/3D_MT/FWD/modelOperator3D.f90:692-800) followed by the V_E
 * weighting of MultA_N (:879-918).  Writes interior edges of out only. */
static void multA_N(const orc_t *o, const cplx *in, int adjt, cplx *out)
{
    int nx = o->nx, ny = o->ny, nz = o->nz;
    double diag_sign = adjt ? -1.0 * ISIGN : (double)ISIGN;
    for (int iz = 2; iz <= nz; iz++)
        for (int iy = 2; iy <= ny; iy++)
            for (int ix = 1; ix <= nx; ix++) {
                long e = IEX(o, ix, iy, iz);
                cplx v = TX(xY, ix, iy) * (in[IEY(o, ix + 1, iy, iz)] - in[IEY(o, ix, iy, iz)] - in[IEY(o, ix + 1, iy - 1, iz)] + in[IEY(o, ix, iy - 1, iz)])
                       + TX(xZ, ix, iz) * (in[IEZ(o, ix + 1, iy, iz)] - in[IEZ(o, ix, iy, iz)] - in[IEZ(o, ix + 1, iy, iz - 1)] + in[IEZ(o, ix, iy, iz - 1)])
                       + o->xXY2[iy] * in[IEX(o, ix, iy + 1, iz)] + o->xXY1[iy] * in[IEX(o, ix, iy - 1, iz)]
                       + o->xXZ2[iz] * in[IEX(o, ix, iy, iz + 1)] + o->xXZ1[iz] * in[IEX(o, ix, iy, iz - 1)]
                       + (TY(xXO, iy, iz) + diag_sign * o->Adiag[e]) * in[e];
                out[e] = v * o->VE[e];
            }
    for (int iz = 2; iz <= nz; iz++)
        for (int iy = 1; iy <= ny; iy++)
            for (int ix = 2; ix <= nx; ix++) {
                long e = IEY(o, ix, iy, iz);
                cplx v = TY(yZ, iy, iz) * (in[IEZ(o, ix, iy + 1, iz)] - in[IEZ(o, ix, iy, iz)] - in[IEZ(o, ix, iy + 1, iz - 1)] + in[IEZ(o, ix, iy, iz - 1)])
                       + TX(yX, ix, iy) * (in[IEX(o, ix, iy + 1, iz)] - in[IEX(o, ix, iy, iz)] - in[IEX(o, ix - 1, iy + 1, iz)] + in[IEX(o, ix - 1, iy, iz)])
                       + o->yYZ2[iz] * in[IEY(o, ix, iy, iz + 1)] + o->yYZ1[iz] * in[IEY(o, ix, iy, iz - 1)]
                       + o->yYX2[ix] * in[IEY(o, ix + 1, iy, iz)] + o->yYX1[ix] * in[IEY(o, ix - 1, iy, iz)]
                       + (TX(yYO, ix, iz) + diag_sign * o->Adiag[e]) * in[e];
                out[e] = v * o->VE[e];
            }
    for (int iz = 1; iz <= nz; iz++)
        for (int iy = 2; iy <= ny; iy++)
            for (int ix = 2; ix <= nx; ix++) {
                long e = IEZ(o, ix, iy, iz);
                cplx v = TX(zX, ix, iz) * (in[IEX(o, ix, iy, iz + 1)] - in[IEX(o, ix, iy, iz)] - in[IEX(o, ix - 1, iy, iz + 1)] + in[IEX(o, ix - 1, iy, iz)])
                       + TY(zY, iy, iz) * (in[IEY(o, ix, iy, iz + 1)] - in[IEY(o, ix, iy, iz)] - in[IEY(o, ix, iy - 1, iz + 1)] + in[IEY(o, ix, iy - 1, iz)])
                       + o->zZX2[ix] * in[IEZ(o, ix + 1, iy, iz)] + o->zZX1[ix] * in[IEZ(o, ix - 1, iy, iz)]
                       + o->zZY2[iy] * in[IEZ(o, ix, iy + 1, iz)] + o->zZY1[iy] * in[IEZ(o, ix, iy - 1, iz)]
                       + (TX(zZO, ix, iy) + diag_sign * o->Adiag[e]) * in[e];
                out[e] = v * o->VE[e];
            }
}

void orc_multA(const orc_t *o, const cplx *in, int adjt, cplx *out) { multA_N(o, in, adjt, out); }

int orc_is_interior_edge(const orc_t *o, long e)
{
    int nx = o->nx, ny = o->ny, nz = o->nz;
    if (e < o->nXe) {
        long j = (e / nx) % (ny + 1), k = e / ((long)nx * (ny + 1));
        return j >= 1 && j <= ny - 1 && k >= 1 && k <= nz - 1;
    }
    e -= o->nXe;
    if (e < o->nYe) {
        long i = e % (nx + 1), k = e / ((long)(nx + 1) * ny);
        return i >= 1 && i <= nx - 1 && k >= 1 && k <= nz - 1;
    }
    e -= o->nYe;
    long i = e % (nx + 1), j = (e / (nx + 1)) % (ny + 1);
    return i >= 1 && i <= nx - 1 && j >= 1 && j <= ny - 1;
}

/* M1solve (f90/3D_MT/FWD/modelOperator3D.f90:1180-1330) */
static void m1solve(const orc_t *o, const cplx *in, int adjt, cplx *out)
{
    int nx = o->nx, ny = o->ny, nz = o->nz;
    const cplx *D = o->Dilu;
    if (!adjt) {
        for (long i = 0; i < o->nE; i++) out[i] = in[i] / o->VE[i];
        for (int ix = 1; ix <= nx; ix++)
            for (int iz = 2; iz <= nz; iz++)
                for (int iy = 2; iy <= ny; iy++) {
                    long e = IEX(o, ix, iy, iz);
                    out[e] = (out[e] - out[IEX(o, ix, iy - 1, iz)] * o->xXY1[iy] - out[IEX(o, ix, iy, iz - 1)] * o->xXZ1[iz]) * D[e];
                }
        for (int iy = 1; iy <= ny; iy++)
            for (int iz = 2; iz <= nz; iz++)
                for (int ix = 2; ix <= nx; ix++) {
                    long e = IEY(o, ix, iy, iz);
                    out[e] = (out[e] - out[IEY(o, ix, iy, iz - 1)] * o->yYZ1[iz] - out[IEY(o, ix - 1, iy, iz)] * o->yYX1[ix]) * D[e];
                }
        for (int iz = 1; iz <= nz; iz++)
            for (int iy = 2; iy <= ny; iy++)
                for (int ix = 2; ix <= nx; ix++) {
                    long e = IEZ(o, ix, iy, iz);
                    out[e] = (out[e] - out[IEZ(o, ix - 1, iy, iz)] * o->zZX1[ix] - out[IEZ(o, ix, iy - 1, iz)] * o->zZY1[iy]) * D[e];
                }
    } else {
        for (int ix = 1; ix <= nx; ix++)
            for (int iy = ny; iy >= 2; iy--)
                for (int iz = nz; iz >= 2; iz--) {
                    long e = IEX(o, ix, iy, iz);
                    out[e] = (in[e] - out[IEX(o, ix, iy + 1, iz)] * o->xXY1[iy + 1] - out[IEX(o, ix, iy, iz + 1)] * o->xXZ1[iz + 1]) * conj(D[e]);
                }
        for (int iy = 1; iy <= ny; iy++)
            for (int ix = nx; ix >= 2; ix--)
                for (int iz = nz; iz >= 2; iz--) {
                    long e = IEY(o, ix, iy, iz);
                    out[e] = (in[e] - out[IEY(o, ix, iy, iz + 1)] * o->yYZ1[iz + 1] - out[IEY(o, ix + 1, iy, iz)] * o->yYX1[ix + 1]) * conj(D[e]);
                }
        for (int iz = 1; iz <= nz; iz++)
            for (int ix = nx; ix >= 2; ix--)
                for (int iy = ny; iy >= 2; iy--) {
                    long e = IEZ(o, ix, iy, iz);
                    out[e] = (in[e] - out[IEZ(o, ix + 1, iy, iz)] * o->zZX1[ix + 1] - out[IEZ(o, ix, iy + 1, iz)] * o->zZY1[iy + 1]) * conj(D[e]);
                }
        for (long i = 0; i < o->nE; i++) out[i] = out[i] / o->VE[i];
    }
}

/* M2solve (f90/3D_MT/FWD/modelOperator3D.f90:1336-1493) */
static void m2solve(const orc_t *o, const cplx *in, int adjt, cplx *out)
{
    int nx = o->nx, ny = o->ny, nz = o->nz;
    const cplx *D = o->Dilu;
    if (!adjt) {
        for (int ix = 1; ix <= nx; ix++)
            for (int iz = nz; iz >= 2; iz--)
                for (int iy = ny; iy >= 2; iy--) {
                    long e = IEX(o, ix, iy, iz);
                    out[e] = in[e] - (out[IEX(o, ix, iy + 1, iz)] * o->xXY2[iy] + out[IEX(o, ix, iy, iz + 1)] * o->xXZ2[iz]) * D[e];
                }
        for (int iy = 1; iy <= ny; iy++)
            for (int iz = nz; iz >= 2; iz--)
                for (int ix = nx; ix >= 2; ix--) {
                    long e = IEY(o, ix, iy, iz);
                    out[e] = in[e] - (out[IEY(o, ix, iy, iz + 1)] * o->yYZ2[iz] + out[IEY(o, ix + 1, iy, iz)] * o->yYX2[ix]) * D[e];
                }
        for (int iz = 1; iz <= nz; iz++)
            for (int iy = ny; iy >= 2; iy--)
                for (int ix = nx; ix >= 2; ix--) {
                    long e = IEZ(o, ix, iy, iz);
                    out[e] = in[e] - (out[IEZ(o, ix + 1, iy, iz)] * o->zZX2[ix] + out[IEZ(o, ix, iy + 1, iz)] * o->zZY2[iy]) * D[e];
                }
    } else {
        for (int ix = 1; ix <= nx; ix++)
            for (int iz = 2; iz <= nz; iz++)
                for (int iy = 2; iy <= ny; iy++) {
                    long e = IEX(o, ix, iy, iz);
                    out[e] = in[e] - out[IEX(o, ix, iy - 1, iz)] * o->xXY2[iy - 1] * conj(D[IEX(o, ix, iy - 1, iz)])
                             - out[IEX(o, ix, iy, iz - 1)] * o->xXZ2[iz - 1] * conj(D[IEX(o, ix, iy, iz - 1)]);
                }
        for (int iy = 1; iy <= ny; iy++)
            for (int iz = 2; iz <= nz; iz++)
                for (int ix = 2; ix <= nx; ix++) {
                    long e = IEY(o, ix, iy, iz);
                    out[e] = in[e] - out[IEY(o, ix, iy, iz - 1)] * o->yYZ2[iz - 1] * conj(D[IEY(o, ix, iy, iz - 1)])
                             - out[IEY(o, ix - 1, iy, iz)] * o->yYX2[ix - 1] * conj(D[IEY(o, ix - 1, iy, iz)]);
                }
        for (int iz = 1; iz <= nz; iz++)
            for (int iy = 2; iy <= ny; iy++)
                for (int ix = 2; ix <= nx; ix++) {
                    long e = IEZ(o, ix, iy, iz);
                    out[e] = in[e] - out[IEZ(o, ix - 1, iy, iz)] * o->zZX2[ix - 1] * conj(D[IEZ(o, ix - 1, iy, iz)])
                             - out[IEZ(o, ix, iy - 1, iz)] * o->zZY2[iy - 1] * conj(D[IEZ(o, ix, iy - 1, iz)]);
                }
    }
}

/* Plane-wise D-ILU variants used to evaluate GPU-parallel alternatives to the
 * natural-ordering recurrence of DiluSetUp/M1solve/M2solve.  Each edge
 * component couples, within the preconditioner, only to its same-component
 * neighbours in the two transverse directions (5-point structure per plane),
 * as in the reference.  For a component the helper returns, for interior edge
 * e, the neighbour indices (-1 if not interior) and the couplings
 *   lo_a = a(e, e-a) (lower, direction a), up_a = a(e, e+a), lo_b, up_b
 * and the plane coordinates (pa, pb) used for the colouring. */
typedef struct { long nb[4]; double cf[4]; int pa, pb; double diagr; } nbrs_t;
static int edge_nbrs(const orc_t *o, long e, nbrs_t *q)
{
    int nx = o->nx, ny = o->ny, nz = o->nz;
    if (!orc_is_interior_edge(o, e)) return 0;
    if (e < o->nXe) {
        int ix = (int)(e % nx) + 1, iy = (int)((e / nx) % (ny + 1)) + 1, iz = (int)(e / ((long)nx * (ny + 1))) + 1;
        q->pa = iy; q->pb = iz;
        q->nb[0] = iy > 2 ? IEX(o, ix, iy - 1, iz) : -1; q->cf[0] = o->xXY1[iy];
        q->nb[1] = iy < ny ? IEX(o, ix, iy + 1, iz) : -1; q->cf[1] = o->xXY2[iy];
        q->nb[2] = iz > 2 ? IEX(o, ix, iy, iz - 1) : -1; q->cf[2] = o->xXZ1[iz];
        q->nb[3] = iz < nz ? IEX(o, ix, iy, iz + 1) : -1; q->cf[3] = o->xXZ2[iz];
        q->diagr = TY(xXO, iy, iz);
    } else if (e < o->nXe + o->nYe) {
        long f = e - o->nXe;
        int ix = (int)(f % (nx + 1)) + 1, iy = (int)((f / (nx + 1)) % ny) + 1, iz = (int)(f / ((long)(nx + 1) * ny)) + 1;
        q->pa = ix; q->pb = iz;
        q->nb[0] = ix > 2 ? IEY(o, ix - 1, iy, iz) : -1; q->cf[0] = o->yYX1[ix];
        q->nb[1] = ix < nx ? IEY(o, ix + 1, iy, iz) : -1; q->cf[1] = o->yYX2[ix];
        q->nb[2] = iz > 2 ? IEY(o, ix, iy, iz - 1) : -1; q->cf[2] = o->yYZ1[iz];
        q->nb[3] = iz < nz ? IEY(o, ix, iy, iz + 1) : -1; q->cf[3] = o->yYZ2[iz];
        q->diagr = TX(yYO, ix, iz);
    } else {
        long f = e - o->nXe - o->nYe;
        int ix = (int)(f % (nx + 1)) + 1, iy = (int)((f / (nx + 1)) % (ny + 1)) + 1, iz = (int)(f / ((long)(nx + 1) * (ny + 1))) + 1;
        q->pa = ix; q->pb = iy;
        q->nb[0] = ix > 2 ? IEZ(o, ix - 1, iy, iz) : -1; q->cf[0] = o->zZX1[ix];
        q->nb[1] = ix < nx ? IEZ(o, ix + 1, iy, iz) : -1; q->cf[1] = o->zZX2[ix];
        q->nb[2] = iy > 2 ? IEZ(o, ix, iy - 1, iz) : -1; q->cf[2] = o->zZY1[iy];
        q->nb[3] = iy < ny ? IEZ(o, ix, iy + 1, iz) : -1; q->cf[3] = o->zZY2[iy];
        q->diagr = TX(zZO, ix, iy);
    }
    return 1;
}
/* coupling from neighbour k back to e: the transpose entry a(nb, e) */
static double back_coef(const orc_t *o, long nbidx, int k)
{
    nbrs_t r;
    edge_nbrs(o, nbidx, &r);
    return r.cf[k ^ 1];  /* lower <-> upper of the same direction */
}
static void rbdilu_setup(orc_t *o, int adjt)
{
    if (!o->Drb) o->Drb = xcalloc(o->nE, sizeof(cplx));
    double ds = adjt ? -1.0 * ISIGN : (double)ISIGN;
    /* red: (pa+pb) even -> D = a_ee; black: D = a_ee - sum a_ej a_je / a_jj */
    for (long e = 0; e < o->nE; e++) {
        nbrs_t q;
        if (!edge_nbrs(o, e, &q)) { o->Drb[e] = 1.0; continue; }
        cplx aee = q.diagr + ds * o->Adiag[e];
        if (((q.pa + q.pb) & 1) == 0) { o->Drb[e] = 1.0 / aee; continue; }
        cplx d = aee;
        for (int k = 0; k < 4; k++) {
            if (q.nb[k] < 0) continue;
            nbrs_t r;
            edge_nbrs(o, q.nb[k], &r);
            cplx ajj = r.diagr + ds * o->Adiag[q.nb[k]];
            d -= q.cf[k] * back_coef(o, q.nb[k], k) / ajj;
        }
        o->Drb[e] = 1.0 / d;
    }
}
/* M^-1 v for M = (D+L) D^-1 (D+U) in red-black order, applied to V_E^-1 v */
static void rbdilu_apply(orc_t *o, const cplx *in, cplx *out)
{
    long n = o->nE;
    cplx *w = xcalloc(n, sizeof(cplx));
    for (long e = 0; e < n; e++) {
        nbrs_t q;
        if (!edge_nbrs(o, e, &q)) continue;
        if (((q.pa + q.pb) & 1) == 0) w[e] = in[e] / o->VE[e] * o->Drb[e];
    }
    for (long e = 0; e < n; e++) {
        nbrs_t q;
        if (!edge_nbrs(o, e, &q)) continue;
        if (((q.pa + q.pb) & 1) == 0) continue;
        cplx s = in[e] / o->VE[e];
        for (int k = 0; k < 4; k++) if (q.nb[k] >= 0) s -= q.cf[k] * w[q.nb[k]];
        w[e] = s * o->Drb[e];
    }
    for (long e = 0; e < n; e++) out[e] = 0.0;
    for (long e = 0; e < n; e++) {
        nbrs_t q;
        if (!edge_nbrs(o, e, &q)) continue;
        if (((q.pa + q.pb) & 1) == 1) { out[e] = w[e]; continue; }
        cplx s = 0.0;
        for (int k = 0; k < 4; k++) if (q.nb[k] >= 0) s += q.cf[k] * w[q.nb[k]];
        out[e] = w[e] - s * o->Drb[e];
    }
    free(w);
}
/* natural-order D-ILU with each triangular solve replaced by nsweep Jacobi
 * sweeps on the triangular system (x <- D^-1 (v - L x)) */
static void dilu_sweep_apply(orc_t *o, const cplx *in, cplx *out)
{
    long n = o->nE;
    cplx *w = xcalloc(n, sizeof(cplx)), *t = xcalloc(n, sizeof(cplx)), *v = xcalloc(n, sizeof(cplx));
    for (long e = 0; e < n; e++) { nbrs_t q; if (edge_nbrs(o, e, &q)) v[e] = in[e] / o->VE[e]; }
    for (long e = 0; e < n; e++) w[e] = v[e] * o->Dilu[e];
    for (int s = 0; s < o->nsweep; s++) {
        for (long e = 0; e < n; e++) {
            nbrs_t q;
            if (!edge_nbrs(o, e, &q)) { t[e] = 0.0; continue; }
            cplx acc = v[e];
            if (q.nb[0] >= 0) acc -= q.cf[0] * w[q.nb[0]];
            if (q.nb[2] >= 0) acc -= q.cf[2] * w[q.nb[2]];
            t[e] = acc * o->Dilu[e];
        }
        memcpy(w, t, n * sizeof(cplx));
    }
    /* (I + D^-1 U) x = w */
    memcpy(out, w, n * sizeof(cplx));
    for (int s = 0; s < o->nsweep; s++) {
        for (long e = 0; e < n; e++) {
            nbrs_t q;
            if (!edge_nbrs(o, e, &q)) { t[e] = 0.0; continue; }
            cplx acc = 0.0;
            if (q.nb[1] >= 0) acc += q.cf[1] * out[q.nb[1]];
            if (q.nb[3] >= 0) acc += q.cf[3] * out[q.nb[3]];
            t[e] = w[e] - acc * o->Dilu[e];
        }
        memcpy(out, t, n * sizeof(cplx));
    }
    free(w); free(t); free(v);
}

/* z-line block-Jacobi preconditioner: for Ex and Ey an exact tridiagonal
 * solve along each vertical line of interior edges (the xXZ / yYZ couplings
 * with the full diagonal), for Ez the diagonal.  M approximates Maxwell;
 * applied to V_E^-1 v.  Not in the reference: a candidate GPU preconditioner
 * (independent lines, coalesced across x). */
static void zline_apply(const orc_t *o, const cplx *in, int adjt, cplx *out)
{
    int nx = o->nx, ny = o->ny, nz = o->nz;
    double ds = adjt ? -1.0 * ISIGN : (double)ISIGN;
    cplx *cp = xcalloc(nz + 2, sizeof(cplx)), *dp = xcalloc(nz + 2, sizeof(cplx));
    for (long i = 0; i < o->nE; i++) out[i] = 0.0;
    for (int comp = 0; comp < 2; comp++) {
        int ilo = comp == 0 ? 1 : 2, ihi = nx, jlo = comp == 0 ? 2 : 1, jhi = comp == 0 ? ny : ny;
        for (int iy = jlo; iy <= jhi; iy++)
            for (int ix = ilo; ix <= ihi; ix++) {
                /* unknowns iz = 2..nz */
                for (int iz = 2; iz <= nz; iz++) {
                    long e = comp == 0 ? IEX(o, ix, iy, iz) : IEY(o, ix, iy, iz);
                    double lo = comp == 0 ? o->xXZ1[iz] : o->yYZ1[iz];
                    double up = comp == 0 ? o->xXZ2[iz] : o->yYZ2[iz];
                    cplx dg = (comp == 0 ? TY(xXO, iy, iz) : TX(yYO, ix, iz)) + ds * o->Adiag[e];
                    cplx rhs = in[e] / o->VE[e];
                    if (iz == 2) { cp[iz] = up / dg; dp[iz] = rhs / dg; }
                    else {
                        cplx den = dg - lo * cp[iz - 1];
                        cp[iz] = up / den;
                        dp[iz] = (rhs - lo * dp[iz - 1]) / den;
                    }
                }
                cplx xn = dp[nz];
                out[comp == 0 ? IEX(o, ix, iy, nz) : IEY(o, ix, iy, nz)] = xn;
                for (int iz = nz - 1; iz >= 2; iz--) {
                    xn = dp[iz] - cp[iz] * xn;
                    out[comp == 0 ? IEX(o, ix, iy, iz) : IEY(o, ix, iy, iz)] = xn;
                }
            }
    }
    for (int iz = 1; iz <= nz; iz++)
        for (int iy = 2; iy <= ny; iy++)
            for (int ix = 2; ix <= nx; ix++) {
                long e = IEZ(o, ix, iy, iz);
                out[e] = in[e] / ((TX(zZO, ix, iy) + ds * o->Adiag[e]) * o->VE[e]);
            }
    free(cp); free(dp);
}

/* Jacobi (diagonal) preconditioner: out = in / diag(V_E * Maxwell) on the
 * interior edges.  Not in the reference; this is the diagonal preconditioner
 * the benchmark configuration names, applied where M1solve+M2solve sit. */
static void jacobi_apply(const orc_t *o, const cplx *in, int adjt, cplx *out)
{
    int nx = o->nx, ny = o->ny, nz = o->nz;
    double diag_sign = adjt ? -1.0 * ISIGN : (double)ISIGN;
    for (long i = 0; i < o->nE; i++) out[i] = 0.0;
    for (int iz = 2; iz <= nz; iz++)
        for (int iy = 2; iy <= ny; iy++)
            for (int ix = 1; ix <= nx; ix++) {
                long e = IEX(o, ix, iy, iz);
                out[e] = in[e] / ((TY(xXO, iy, iz) + diag_sign * o->Adiag[e]) * o->VE[e]);
            }
    for (int iz = 2; iz <= nz; iz++)
        for (int iy = 1; iy <= ny; iy++)
            for (int ix = 2; ix <= nx; ix++) {
                long e = IEY(o, ix, iy, iz);
                out[e] = in[e] / ((TX(yYO, ix, iz) + diag_sign * o->Adiag[e]) * o->VE[e]);
            }
    for (int iz = 1; iz <= nz; iz++)
        for (int iy = 2; iy <= ny; iy++)
            for (int ix = 2; ix <= nx; ix++) {
                long e = IEZ(o, ix, iy, iz);
                out[e] = in[e] / ((TX(zZO, ix, iy) + diag_sign * o->Adiag[e]) * o->VE[e]);
            }
}

/* DivCgrad (f90/3D_MT/FWD/modelOperator3D.f90:1760-1810) */
static void divcgrad(const orc_t *o, const cplx *in, cplx *out)
{
    int nx = o->nx, ny = o->ny, nz = o->nz;
    for (int iz = 2; iz <= nz; iz++)
        for (int iy = 2; iy <= ny; iy++)
            for (int ix = 2; ix <= nx; ix++) {
                out[IND(o, ix, iy, iz)] = in[IND(o, ix + 1, iy, iz)] * o->db2[IEX(o, ix, iy, iz)]
                    + in[IND(o, ix - 1, iy, iz)] * o->db1[IEX(o, ix, iy, iz)]
                    + in[IND(o, ix, iy + 1, iz)] * o->db2[IEY(o, ix, iy, iz)]
                    + in[IND(o, ix, iy - 1, iz)] * o->db1[IEY(o, ix, iy, iz)]
                    + in[IND(o, ix, iy, iz + 1)] * o->db2[IEZ(o, ix, iy, iz)]
                    + in[IND(o, ix, iy, iz - 1)] * o->db1[IEZ(o, ix, iy, iz)]
                    + in[IND(o, ix, iy, iz)] * o->c[IND(o, ix, iy, iz)];
            }
}

/* DivCgradILU (f90/3D_MT/FWD/modelOperator3D.f90:1690-1755) */
static void divcgrad_ilu(const orc_t *o, const cplx *in, cplx *out)
{
    int nx = o->nx, ny = o->ny, nz = o->nz;
    for (long i = 0; i < o->nN; i++) out[i] = 0.0;
    for (int iz = 2; iz <= nz; iz++)
        for (int iy = 2; iy <= ny; iy++)
            for (int ix = 2; ix <= nx; ix++)
                out[IND(o, ix, iy, iz)] = in[IND(o, ix, iy, iz)]
                    - out[IND(o, ix - 1, iy, iz)] * o->db1[IEX(o, ix, iy, iz)] * o->d[IND(o, ix - 1, iy, iz)]
                    - out[IND(o, ix, iy - 1, iz)] * o->db1[IEY(o, ix, iy, iz)] * o->d[IND(o, ix, iy - 1, iz)]
                    - out[IND(o, ix, iy, iz - 1)] * o->db1[IEZ(o, ix, iy, iz)] * o->d[IND(o, ix, iy, iz - 1)];
    for (int iz = nz; iz >= 2; iz--)
        for (int iy = ny; iy >= 2; iy--)
            for (int ix = nx; ix >= 2; ix--)
                out[IND(o, ix, iy, iz)] = (out[IND(o, ix, iy, iz)]
                    - out[IND(o, ix + 1, iy, iz)] * o->db2[IEX(o, ix, iy, iz)]
                    - out[IND(o, ix, iy + 1, iz)] * o->db2[IEY(o, ix, iy, iz)]
                    - out[IND(o, ix, iy, iz + 1)] * o->db2[IEZ(o, ix, iy, iz)]) * o->d[IND(o, ix, iy, iz)];
}

/* Jacobi preconditioner for the div-correction Poisson system (node-wise
 * 1/c on interior nodes); the GPU path uses it in place of DivCgradILU. */
static void divcgrad_jacobi(const orc_t *o, const cplx *in, cplx *out)
{
    int nx = o->nx, ny = o->ny, nz = o->nz;
    for (long i = 0; i < o->nN; i++) out[i] = 0.0;
    for (int iz = 2; iz <= nz; iz++)
        for (int iy = 2; iy <= ny; iy++)
            for (int ix = 2; ix <= nx; ix++) {
                long n = IND(o, ix, iy, iz);
                out[n] = in[n] / o->c[n];
            }
}

/* DivC (f90/3D_MT/FWD/modelOperator3D.f90:1817-1925) */
static void divc(const orc_t *o, const cplx *E, cplx *out)
{
    int nx = o->nx, ny = o->ny, nz = o->nz, nzAir = o->nzAir;
    const double *s = o->sigE;
    for (int ix = 2; ix <= nx; ix++)
        for (int iy = 2; iy <= ny; iy++) {
            double rx = 1.0 / o->delX[ix], ry = 1.0 / o->delY[iy];
            for (int iz = 2; iz <= nzAir; iz++) {
                double rz = 1.0 / o->delZ[iz];
                out[IND(o, ix, iy, iz)] = SIGMA_AIR * (E[IEX(o, ix, iy, iz)] - E[IEX(o, ix - 1, iy, iz)]) * rx
                    + SIGMA_AIR * (E[IEY(o, ix, iy, iz)] - E[IEY(o, ix, iy - 1, iz)]) * ry
                    + SIGMA_AIR * (E[IEZ(o, ix, iy, iz)] - E[IEZ(o, ix, iy, iz - 1)]) * rz;
            }
            int iz = nzAir + 1;
            {
                double rz = 1.0 / o->delZ[iz];
                out[IND(o, ix, iy, iz)] = (s[IEX(o, ix, iy, iz)] * E[IEX(o, ix, iy, iz)] - s[IEX(o, ix - 1, iy, iz)] * E[IEX(o, ix - 1, iy, iz)]) * rx
                    + (s[IEY(o, ix, iy, iz)] * E[IEY(o, ix, iy, iz)] - s[IEY(o, ix, iy - 1, iz)] * E[IEY(o, ix, iy - 1, iz)]) * ry
                    + (s[IEZ(o, ix, iy, iz)] * E[IEZ(o, ix, iy, iz)] - SIGMA_AIR * E[IEZ(o, ix, iy, iz - 1)]) * rz;
            }
            for (iz = nzAir + 2; iz <= nz; iz++) {
                double rz = 1.0 / o->delZ[iz];
                out[IND(o, ix, iy, iz)] = (s[IEX(o, ix, iy, iz)] * E[IEX(o, ix, iy, iz)] - s[IEX(o, ix - 1, iy, iz)] * E[IEX(o, ix - 1, iy, iz)]) * rx
                    + (s[IEY(o, ix, iy, iz)] * E[IEY(o, ix, iy, iz)] - s[IEY(o, ix, iy - 1, iz)] * E[IEY(o, ix, iy - 1, iz)]) * ry
                    + (s[IEZ(o, ix, iy, iz)] * E[IEZ(o, ix, iy, iz)] - s[IEZ(o, ix, iy, iz - 1)] * E[IEZ(o, ix, iy, iz - 1)]) * rz;
            }
        }
}

/* Div (f90/FIELDS/FiniteDiff3D/sg_diff_oper.f90:26-93), edge -> node */
static void div_plain(const orc_t *o, const cplx *E, cplx *out)
{
    int nx = o->nx, ny = o->ny, nz = o->nz;
    for (int ix = 2; ix <= nx; ix++)
        for (int iy = 2; iy <= ny; iy++)
            for (int iz = 2; iz <= nz; iz++)
                out[IND(o, ix, iy, iz)] = (E[IEX(o, ix, iy, iz)] - E[IEX(o, ix - 1, iy, iz)]) / o->delX[ix]
                    + (E[IEY(o, ix, iy, iz)] - E[IEY(o, ix, iy - 1, iz)]) / o->delY[iy]
                    + (E[IEZ(o, ix, iy, iz)] - E[IEZ(o, ix, iy, iz - 1)]) / o->delZ[iz];
}

/* Grad (f90/FIELDS/FiniteDiff3D/sg_diff_oper.f90:98-200): node -> interior edges */
static void grad_sub(const orc_t *o, const cplx *phi, cplx *E)
{
    int nx = o->nx, ny = o->ny, nz = o->nz;
    for (int ix = 1; ix <= nx; ix++)
        for (int iy = 2; iy <= ny; iy++)
            for (int iz = 2; iz <= nz; iz++)
                E[IEX(o, ix, iy, iz)] -= (phi[IND(o, ix + 1, iy, iz)] - phi[IND(o, ix, iy, iz)]) / o->dx[ix];
    for (int ix = 2; ix <= nx; ix++)
        for (int iy = 1; iy <= ny; iy++)
            for (int iz = 2; iz <= nz; iz++)
                E[IEY(o, ix, iy, iz)] -= (phi[IND(o, ix, iy + 1, iz)] - phi[IND(o, ix, iy, iz)]) / o->dy[iy];
    for (int ix = 2; ix <= nx; ix++)
        for (int iy = 2; iy <= ny; iy++)
            for (int iz = 1; iz <= nz; iz++)
                E[IEZ(o, ix, iy, iz)] -= (phi[IND(o, ix, iy, iz + 1)] - phi[IND(o, ix, iy, iz)]) / o->dz[iz];
}

void orc_divc(const orc_t *o, const cplx *E, cplx *out)
{
    for (long i = 0; i < o->nN; i++) out[i] = 0.0;
    divc(o, E, out);
}
void orc_divcgrad(const orc_t *o, const cplx *in, cplx *out)
{
    for (long i = 0; i < o->nN; i++) out[i] = 0.0;
    divcgrad(o, in, out);
}

/* ------------------------------------------------------------------------ */
/* BLAS-1 helpers                                                            */
/* ------------------------------------------------------------------------ */
static cplx dotc(const cplx *a, const cplx *b, long n)
{
    cplx s = 0.0;
    for (long i = 0; i < n; i++) s += conj(a[i]) * b[i];
    return s;
}
static double nrm(const cplx *a, long n) { return sqrt(creal(dotc(a, a, n))); }

/* ------------------------------------------------------------------------ */
/* Krylov solvers                                                            */
/* ------------------------------------------------------------------------ */
typedef struct {
    int maxIt;
    double tol;
    int niter;
    double *rerr;
    int failed;
} kss_t;

/* PCG (f90/3D_MT/FWD/solver.f90:40-118) on node scalars */
static void pcg(const orc_t *o, const cplx *b, cplx *x, kss_t *it)
{
    long n = o->nN;
    cplx *r = xcalloc(n, sizeof(cplx)), *s = xcalloc(n, sizeof(cplx));
    cplx *p = xcalloc(n, sizeof(cplx)), *q = xcalloc(n, sizeof(cplx));
    cplx delta, deltaOld = 1.0, beta, alpha;
    divcgrad(o, x, r);
    for (long i = 0; i < n; i++) r[i] = b[i] - r[i];
    double bnorm = nrm(b, n), rnorm = nrm(r, n);
    int i = 1;
    it->rerr[0] = rnorm / bnorm;
    while (it->rerr[i - 1] > it->tol && i < it->maxIt) {
        if (o->precond == ORC_PC_DILU) divcgrad_ilu(o, r, s);
        else divcgrad_jacobi(o, r, s);
        delta = dotc(r, s, n);
        if (i == 1) {
            for (long k = 0; k < n; k++) p[k] = s[k];
        } else {
            beta = delta / deltaOld;
            for (long k = 0; k < n; k++) p[k] = s[k] + beta * p[k];
        }
        divcgrad(o, p, q);
        alpha = delta / dotc(p, q, n);
        for (long k = 0; k < n; k++) x[k] += alpha * p[k];
        for (long k = 0; k < n; k++) r[k] += -alpha * q[k];
        deltaOld = delta;
        i++;
        rnorm = nrm(r, n);
        it->rerr[i - 1] = rnorm / bnorm;
    }
    it->niter = i;
    free(r); free(s); free(p); free(q);
}

static void precond_L(const orc_t *o, const cplx *in, int adjt, cplx *out)
{
    if (o->precond == ORC_PC_DILU) m1solve(o, in, adjt, out);
    else if (o->precond == ORC_PC_RBDILU) rbdilu_apply((orc_t *)o, in, out);
    else if (o->precond == ORC_PC_DILU_SWEEP) dilu_sweep_apply((orc_t *)o, in, out);
    else if (o->precond == ORC_PC_ZLINE) zline_apply(o, in, adjt, out);
    else jacobi_apply(o, in, adjt, out);
}
static void precond_U(const orc_t *o, const cplx *in, int adjt, cplx *out)
{
    if (o->precond == ORC_PC_DILU) m2solve(o, in, adjt, out);
    else for (long i = 0; i < o->nE; i++) out[i] = in[i];
}

/* QMR without look-ahead (f90/3D_MT/FWD/solver.f90:122-343) */
static void qmr(const orc_t *o, const cplx *b, cplx *x, kss_t *it)
{
    long n = o->nE;
    cplx *R = xcalloc(n, sizeof(cplx)), *VT = xcalloc(n, sizeof(cplx)), *Y = xcalloc(n, sizeof(cplx));
    cplx *Z = xcalloc(n, sizeof(cplx)), *WT = xcalloc(n, sizeof(cplx)), *V = xcalloc(n, sizeof(cplx));
    cplx *W = xcalloc(n, sizeof(cplx)), *YT = xcalloc(n, sizeof(cplx)), *ZT = xcalloc(n, sizeof(cplx));
    cplx *P = xcalloc(n, sizeof(cplx)), *Q = xcalloc(n, sizeof(cplx)), *PT = xcalloc(n, sizeof(cplx));
    cplx *D = xcalloc(n, sizeof(cplx)), *S = xcalloc(n, sizeof(cplx));
    cplx ETA, PDE, EPSIL = 0, RDE, BETA, DELTA, RHO, PSI, RHO1, GAMM, GAMM1, THET = 0, THET1 = 0, TM2;
    multA_N(o, x, 0, R);
    for (long i = 0; i < n; i++) R[i] = b[i] - R[i];
    cplx bnorm = csqrt(dotc(b, b, n)), rnorm = csqrt(dotc(R, R, n));
    if (isnan(cabs(bnorm))) { it->failed = 1; it->niter = 0; goto done; }
    int iter = 1;
    it->rerr[0] = creal(rnorm / bnorm);
    memcpy(VT, R, n * sizeof(cplx));
    precond_L(o, VT, 0, Y);
    RHO = csqrt(dotc(Y, Y, n));
    memcpy(WT, R, n * sizeof(cplx));
    precond_U(o, WT, 1, Z);
    PSI = csqrt(dotc(Z, Z, n));
    GAMM = 1.0;
    ETA = -1.0;
    while (it->rerr[iter - 1] > it->tol && iter < it->maxIt) {
        if (RHO == 0.0 || PSI == 0.0) { it->failed = 1; break; }
        cplx rhoInv = (1.0 / RHO), psiInv = (1.0 / PSI);
        for (long i = 0; i < n; i++) {
            V[i] = rhoInv * VT[i];
            W[i] = psiInv * WT[i];
            Y[i] = rhoInv * Y[i];
            Z[i] = psiInv * Z[i];
        }
        DELTA = dotc(Z, Y, n);
        if (DELTA == 0.0) { it->failed = 1; break; }
        precond_U(o, Y, 0, YT);
        precond_L(o, Z, 1, ZT);
        if (iter == 1) {
            memcpy(P, YT, n * sizeof(cplx));
            memcpy(Q, ZT, n * sizeof(cplx));
        } else {
            PDE = -PSI * DELTA / EPSIL;
            RDE = -RHO * conj(DELTA / EPSIL);
            for (long i = 0; i < n; i++) {
                P[i] = YT[i] + PDE * P[i];
                Q[i] = ZT[i] + RDE * Q[i];
            }
        }
        multA_N(o, P, 0, PT);
        EPSIL = dotc(Q, PT, n);
        if (EPSIL == 0.0) { it->failed = 1; break; }
        BETA = EPSIL / DELTA;
        if (BETA == 0.0) { it->failed = 1; break; }
        for (long i = 0; i < n; i++) VT[i] = PT[i] - BETA * V[i];
        RHO1 = RHO;
        precond_L(o, VT, 0, Y);
        RHO = csqrt(dotc(Y, Y, n));
        multA_N(o, Q, 1, WT);
        for (long i = 0; i < n; i++) WT[i] += -conj(BETA) * W[i];
        precond_U(o, WT, 1, Z);
        PSI = csqrt(dotc(Z, Z, n));
        if (iter > 1) THET1 = THET;
        THET = RHO / (GAMM * cabs(BETA));
        GAMM1 = GAMM;
        GAMM = 1.0 / csqrt(1.0 + THET * THET);
        if (GAMM == 0.0) break;
        ETA = -ETA * RHO1 * GAMM * GAMM / (BETA * GAMM1 * GAMM1);
        if (iter == 1) {
            for (long i = 0; i < n; i++) { D[i] = ETA * P[i]; S[i] = ETA * PT[i]; }
        } else {
            TM2 = THET1 * THET1 * GAMM * GAMM;
            for (long i = 0; i < n; i++) {
                D[i] = ETA * P[i] + TM2 * D[i];
                S[i] = ETA * PT[i] + TM2 * S[i];
            }
        }
        for (long i = 0; i < n; i++) { x[i] += D[i]; R[i] -= S[i]; }
        rnorm = csqrt(dotc(R, R, n));
        iter++;
        it->rerr[iter - 1] = creal(rnorm / bnorm);
    }
    it->niter = iter;
done:
    free(R); free(VT); free(Y); free(Z); free(WT); free(V); free(W); free(YT); free(ZT);
    free(P); free(Q); free(PT); free(D); free(S);
}

/* BiCGStab (f90/3D_MT/FWD/solver.f90:346-555).  One deviation: the best
 * iterate xmin starts from the initial guess, where the MF routine leaves it
 * as the zero vector it was created as (a reference defect that returns a
 * zero field when no iterate improves on the initial residual). */
static void bicg(const orc_t *o, const cplx *b, cplx *x, kss_t *it)
{
    long n = o->nE;
    double bnorm = nrm(b, n);
    if (isnan(bnorm)) { it->failed = 1; it->niter = 0; return; }
    if (bnorm == 0.0) {
        memcpy(x, b, n * sizeof(cplx));
        it->niter = 1; it->failed = 0;
        for (int i = 0; i < it->maxIt; i++) it->rerr[i] = 0.0;
        return;
    }
    cplx *R = xcalloc(n, sizeof(cplx)), *RT = xcalloc(n, sizeof(cplx)), *V = xcalloc(n, sizeof(cplx));
    cplx *T = xcalloc(n, sizeof(cplx)), *P = xcalloc(n, sizeof(cplx)), *PT = xcalloc(n, sizeof(cplx));
    cplx *PH = xcalloc(n, sizeof(cplx)), *S = xcalloc(n, sizeof(cplx)), *ST = xcalloc(n, sizeof(cplx));
    cplx *SH = xcalloc(n, sizeof(cplx)), *xhalf = xcalloc(n, sizeof(cplx)), *xmin = xcalloc(n, sizeof(cplx));
    multA_N(o, x, 0, R);
    for (long i = 0; i < n; i++) R[i] = b[i] - R[i];
    double rnorm = nrm(R, n);
    double btol = it->tol * bnorm;
    if (rnorm <= btol) {
        it->niter = 1; it->failed = 0; it->rerr[0] = rnorm / bnorm;
        goto done;
    }
    double rnormin = rnorm;
    it->rerr[0] = rnormin / bnorm;
    int converged = 0, imin = 0;
    cplx RHO = 1.0, RHO1, OMEGA = 1.0, ALPHA = 0.0, BETA, RTV, TT;
    memcpy(RT, R, n * sizeof(cplx));
    memcpy(xmin, x, n * sizeof(cplx));
    for (int iter = 1; iter <= it->maxIt; iter++) {
        RHO1 = RHO;
        RHO = dotc(RT, R, n);
        if (RHO == 0.0) { it->failed = 1; break; }
        if (iter == 1) {
            memcpy(P, R, n * sizeof(cplx));
        } else {
            BETA = (RHO / RHO1) * (ALPHA / OMEGA);
            if (BETA == 0.0) { it->failed = 1; break; }
            for (long i = 0; i < n; i++) P[i] = P[i] - OMEGA * V[i];
            for (long i = 0; i < n; i++) P[i] = R[i] + BETA * P[i];
        }
        precond_L(o, P, 0, PT);
        precond_U(o, PT, 0, PH);
        multA_N(o, PH, 0, V);
        RTV = dotc(RT, V, n);
        if (RTV == 0.0) { it->failed = 1; break; }
        ALPHA = RHO / RTV;
        if (ALPHA == 0.0) { it->failed = 1; break; }
        for (long i = 0; i < n; i++) xhalf[i] = x[i] + ALPHA * PH[i];
        for (long i = 0; i < n; i++) S[i] = R[i] - ALPHA * V[i];
        precond_L(o, S, 0, ST);
        precond_U(o, ST, 0, SH);
        multA_N(o, SH, 0, T);
        TT = dotc(T, T, n);
        if (TT == 0.0) { it->failed = 1; break; }
        OMEGA = dotc(T, S, n) / TT;
        if (OMEGA == 0.0) { it->failed = 1; break; }
        for (long i = 0; i < n; i++) x[i] = xhalf[i] + OMEGA * SH[i];
        for (long i = 0; i < n; i++) R[i] = S[i] - OMEGA * T[i];
        rnorm = nrm(R, n);
        it->rerr[iter - 1] = rnorm / bnorm;
        if (rnorm < btol) {
            it->failed = 0; it->niter = iter; converged = 1;
            break;
        }
        if (rnorm < rnormin) {
            rnormin = rnorm;
            memcpy(xmin, x, n * sizeof(cplx));
            imin = iter;
        }
    }
    if (!converged) {
        memcpy(x, xmin, n * sizeof(cplx));
        it->niter = it->maxIt;
        if (imin > 0) it->rerr[it->maxIt - 1] = it->rerr[imin - 1];
        else it->rerr[it->maxIt - 1] = it->rerr[0];
    }
done:
    free(R); free(RT); free(V); free(T); free(P); free(PT); free(PH); free(S); free(ST); free(SH);
    free(xhalf); free(xmin);
}

/* Bi-CG for the complex-symmetric system (A^T = A) with the shadow residual
 * conj(r0), which reduces to the conjugate-orthogonal CG (COCG, van der Vorst &
 * Melissen 1990): one operator application per iteration; bilinear (not
 * conjugated) products.  Preconditioned with the (complex-symmetric) diagonal
 * or D-ILU preconditioner applied as z = M^-1 r.  Returns like bicg(): the
 * best iterate when not converged. */
static cplx dotu(const cplx *a, const cplx *b, long n)
{
    cplx s = 0.0;
    for (long i = 0; i < n; i++) s += a[i] * b[i];
    return s;
}
static void cocg(const orc_t *o, const cplx *b, cplx *x, kss_t *it)
{
    long n = o->nE;
    double bnorm = nrm(b, n);
    if (isnan(bnorm)) { it->failed = 1; it->niter = 0; return; }
    if (bnorm == 0.0) {
        memcpy(x, b, n * sizeof(cplx));
        it->niter = 1; it->failed = 0;
        for (int i = 0; i < it->maxIt; i++) it->rerr[i] = 0.0;
        return;
    }
    cplx *R = xcalloc(n, sizeof(cplx)), *Z = xcalloc(n, sizeof(cplx)), *P = xcalloc(n, sizeof(cplx));
    cplx *Q = xcalloc(n, sizeof(cplx)), *T = xcalloc(n, sizeof(cplx)), *xmin = xcalloc(n, sizeof(cplx));
    multA_N(o, x, 0, R);
    for (long i = 0; i < n; i++) R[i] = b[i] - R[i];
    double rnorm = nrm(R, n), btol = it->tol * bnorm, rnormin = rnorm;
    it->rerr[0] = rnorm / bnorm;
    memcpy(xmin, x, n * sizeof(cplx));
    int converged = 0, imin = 0;
    if (rnorm <= btol) { it->niter = 1; it->failed = 0; goto done; }
    precond_L(o, R, 0, T);
    precond_U(o, T, 0, Z);
    memcpy(P, Z, n * sizeof(cplx));
    cplx rho = dotu(R, Z, n);
    for (int iter = 1; iter <= it->maxIt; iter++) {
        multA_N(o, P, 0, Q);
        cplx mu = dotu(P, Q, n);
        if (mu == 0.0 || rho == 0.0) { it->failed = 1; break; }
        cplx alpha = rho / mu;
        for (long i = 0; i < n; i++) { x[i] += alpha * P[i]; R[i] -= alpha * Q[i]; }
        rnorm = nrm(R, n);
        it->rerr[iter - 1] = rnorm / bnorm;
        if (rnorm < btol) { it->niter = iter; converged = 1; break; }
        if (rnorm < rnormin) { rnormin = rnorm; memcpy(xmin, x, n * sizeof(cplx)); imin = iter; }
        precond_L(o, R, 0, T);
        precond_U(o, T, 0, Z);
        cplx rho_new = dotu(R, Z, n);
        cplx beta = rho_new / rho;
        rho = rho_new;
        for (long i = 0; i < n; i++) P[i] = Z[i] + beta * P[i];
    }
    if (!converged) {
        memcpy(x, xmin, n * sizeof(cplx));
        it->niter = it->maxIt;
        it->rerr[it->maxIt - 1] = imin > 0 ? it->rerr[imin - 1] : it->rerr[0];
    }
done:
    free(R); free(Z); free(P); free(Q); free(T); free(xmin);
}

/* ------------------------------------------------------------------------ */
/* divergence correction and the solve driver                                */
/* ------------------------------------------------------------------------ */

/* SdivCorr (f90/3D_MT/FWD/EMsolve3D.f90:403-492), in place on E */
static void sdivcorr(orc_t *o, cplx *E, const cplx *phi0)
{
    long nN = o->nN;
    kss_t it = {0};
    it.maxIt = o->MaxIterDivCor;
    it.tol = o->tolDivCor;
    it.rerr = xcalloc(it.maxIt, sizeof(double));
    cplx *phiSol = xcalloc(nN, sizeof(cplx)), *phiRHS = xcalloc(nN, sizeof(cplx));
    divc(o, E, phiRHS);
    if (phi0) for (long i = 0; i < nN; i++) phiRHS[i] = phiRHS[i] - phi0[i];
    int k = o->nDivCor - 1;
    o->divJ[2 * k] = sqrt(creal(dotc(phiRHS, phiRHS, nN)));
    for (long i = 0; i < nN; i++) phiRHS[i] = o->VN[i] * phiRHS[i];
    pcg(o, phiRHS, phiSol, &it);
    memcpy(&o->DivCorRelErr[(size_t)k * o->MaxIterDivCor], it.rerr, sizeof(double) * it.maxIt);
    o->DivCorIters[k] = it.niter;
    grad_sub(o, phiSol, E);
    for (long i = 0; i < nN; i++) phiRHS[i] = 0.0;
    divc(o, E, phiRHS);
    if (phi0) for (long i = 0; i < nN; i++) phiRHS[i] = phiRHS[i] - phi0[i];
    o->divJ[2 * k + 1] = sqrt(creal(dotc(phiRHS, phiRHS, nN)));
    free(phiSol); free(phiRHS); free(it.rerr);
}

/* AdjtBC (f90/3D_MT/FWD/modelOperator3D.f90:920-1057): boundary values of the
 * transpose solution, A_IB^T e, written into the boundary edges of bc (a full
 * edge vector; interior entries untouched).  The face arrays are applied in
 * the order copy_bcvector (f90/FIELDS/FiniteDiff3D/sg_boundary.f90:1095-1201)
 * writes them, so edges shared by two faces take the later face's value. */
static void adjt_bc(const orc_t *o, const cplx *E, cplx *bc)
{
    int nx = o->nx, ny = o->ny, nz = o->nz;
    /* xYmin/xYmax: Ex on iy = 1, ny+1 */
    for (int ix = 1; ix <= nx; ix++) {
        bc[IEX(o, ix, 1, 1)] = 0; bc[IEX(o, ix, ny + 1, 1)] = 0;
        bc[IEX(o, ix, 1, nz + 1)] = 0; bc[IEX(o, ix, ny + 1, nz + 1)] = 0;
        for (int iz = 2; iz <= nz; iz++) {
            bc[IEX(o, ix, 1, iz)] = -TX(yX, ix, 1) * E[IEY(o, ix, 1, iz)] + TX(yX, ix + 1, 1) * E[IEY(o, ix + 1, 1, iz)] + o->xXY1[2] * E[IEX(o, ix, 2, iz)];
            bc[IEX(o, ix, ny + 1, iz)] = TX(yX, ix, ny) * E[IEY(o, ix, ny, iz)] - TX(yX, ix + 1, ny) * E[IEY(o, ix + 1, ny, iz)] + o->xXY2[ny] * E[IEX(o, ix, ny, iz)];
        }
    }
    /* zYmin/zYmax: Ez on iy = 1, ny+1 */
    for (int iz = 1; iz <= nz; iz++) {
        bc[IEZ(o, 1, 1, iz)] = 0; bc[IEZ(o, 1, ny + 1, iz)] = 0;
        bc[IEZ(o, nx + 1, 1, iz)] = 0; bc[IEZ(o, nx + 1, ny + 1, iz)] = 0;
        for (int ix = 2; ix <= nx; ix++) {
            bc[IEZ(o, ix, 1, iz)] = -TY(yZ, 1, iz) * E[IEY(o, ix, 1, iz)] + TY(yZ, 1, iz + 1) * E[IEY(o, ix, 1, iz + 1)] + o->zZY1[2] * E[IEZ(o, ix, 2, iz)];
            bc[IEZ(o, ix, ny + 1, iz)] = TY(yZ, ny, iz) * E[IEY(o, ix, ny, iz)] - TY(yZ, ny, iz + 1) * E[IEY(o, ix, ny, iz + 1)] + o->zZY2[ny] * E[IEZ(o, ix, ny, iz)];
        }
    }
    /* yXmin/yXmax: Ey on ix = 1, nx+1 */
    for (int iy = 1; iy <= ny; iy++) {
        bc[IEY(o, nx + 1, iy, 1)] = 0; bc[IEY(o, 1, iy, 1)] = 0;
        bc[IEY(o, nx + 1, iy, nz + 1)] = 0; bc[IEY(o, 1, iy, nz + 1)] = 0;
        for (int iz = 2; iz <= nz; iz++) {
            bc[IEY(o, nx + 1, iy, iz)] = TX(xY, nx, iy) * E[IEX(o, nx, iy, iz)] - TX(xY, nx, iy + 1) * E[IEX(o, nx, iy + 1, iz)] + o->yYX2[nx] * E[IEY(o, nx, iy, iz)];
            bc[IEY(o, 1, iy, iz)] = -TX(xY, 1, iy) * E[IEX(o, 1, iy, iz)] + TX(xY, 1, iy + 1) * E[IEX(o, 1, iy + 1, iz)] + o->yYX1[2] * E[IEY(o, 2, iy, iz)];
        }
    }
    /* zXmin/zXmax: Ez on ix = 1, nx+1 */
    for (int iz = 1; iz <= nz; iz++) {
        bc[IEZ(o, nx + 1, 1, iz)] = 0; bc[IEZ(o, 1, 1, iz)] = 0;
        bc[IEZ(o, nx + 1, ny + 1, iz)] = 0; bc[IEZ(o, 1, ny + 1, iz)] = 0;
        for (int iy = 2; iy <= ny; iy++) {
            bc[IEZ(o, nx + 1, iy, iz)] = TX(xZ, nx, iz) * E[IEX(o, nx, iy, iz)] - TX(xZ, nx, iz + 1) * E[IEX(o, nx, iy, iz + 1)] + o->zZX2[nx] * E[IEZ(o, nx, iy, iz)];
            bc[IEZ(o, 1, iy, iz)] = -TX(xZ, 1, iz) * E[IEX(o, 1, iy, iz)] + TX(xZ, 1, iz + 1) * E[IEX(o, 1, iy, iz + 1)] + o->zZX1[2] * E[IEZ(o, 2, iy, iz)];
        }
    }
    /* xZmin/xZmax: Ex on iz = 1, nz+1 */
    for (int ix = 1; ix <= nx; ix++) {
        bc[IEX(o, ix, 1, 1)] = 0; bc[IEX(o, ix, 1, nz + 1)] = 0;
        bc[IEX(o, ix, ny + 1, 1)] = 0; bc[IEX(o, ix, ny + 1, nz + 1)] = 0;
        for (int iy = 2; iy <= ny; iy++) {
            bc[IEX(o, ix, iy, 1)] = -TX(zX, ix, 1) * E[IEZ(o, ix, iy, 1)] + TX(zX, ix + 1, 1) * E[IEZ(o, ix + 1, iy, 1)] + o->xXZ1[2] * E[IEX(o, ix, iy, 2)];
            bc[IEX(o, ix, iy, nz + 1)] = TX(zX, ix, nz) * E[IEZ(o, ix, iy, nz)] - TX(zX, ix + 1, nz) * E[IEZ(o, ix + 1, iy, nz)] + o->xXZ2[nz] * E[IEX(o, ix, iy, nz)];
        }
    }
    /* yZmin/yZmax: Ey on iz = 1, nz+1.  The reference zeroes yZmin(:,1),
     * yZmax(:,1) and yZmin(nx+1,:) before the loop and never sets yZmin(1,:),
     * yZmax(1,:) or yZmax(nx+1,:), which therefore keep the zero they were
     * created with. */
    for (int iy = 1; iy <= ny; iy++) {
        bc[IEY(o, 1, iy, 1)] = 0; bc[IEY(o, nx + 1, iy, 1)] = 0;
        bc[IEY(o, 1, iy, nz + 1)] = 0; bc[IEY(o, nx + 1, iy, nz + 1)] = 0;
        for (int ix = 2; ix <= nx; ix++) {
            bc[IEY(o, ix, iy, 1)] = -TY(zY, iy, 1) * E[IEZ(o, ix, iy, 1)] + TY(zY, iy + 1, 1) * E[IEZ(o, ix, iy + 1, 1)] + o->yYZ1[2] * E[IEY(o, ix, iy, 2)];
            bc[IEY(o, ix, iy, nz + 1)] = TY(zY, iy, nz) * E[IEZ(o, ix, iy, nz)] - TY(zY, iy + 1, nz) * E[IEZ(o, ix, iy + 1, nz)] + o->yYZ2[nz] * E[IEY(o, ix, iy, nz)];
        }
    }
}

void orc_adjt_bc(const orc_t *o, const cplx *E, cplx *bc) { adjt_bc(o, E, bc); }

/* FWDsolve3D (f90/3D_MT/FWD/EMsolve3D.f90:116-391).
 *   trans = 0: forward problem.  bc (full edge vector, boundary entries used)
 *              gives the tangential boundary field; src (optional, full edge
 *              vector) is an interior source already multiplied by
 *              -ISIGN*i*omega*mu0.
 *   trans = 1: transposed problem, src is the (V_E-weighted) adjoint source;
 *              bc (optional) the boundary data.
 *   e: full edge vector, solution on output (interior initial guess on input
 *      is ignored, as in the reference, which zeroes the boundary only; the
 *      interior of e on input is used as the initial guess).
 * Returns 0 converged, 1 not converged / failed.
 */
int orc_fwdsolve(orc_t *o, int trans, const cplx *bc, const cplx *src, cplx *e)
{
    long nE = o->nE, nN = o->nN;
    cplx *b = xcalloc(nE, sizeof(cplx)), *temp = xcalloc(nE, sizeof(cplx));
    cplx *phi0 = NULL;
    cplx i_omega_mu = CMPLX(0.0, 1.0 * ISIGN * MU_0 * o->omega);
    o->nIterTotal = 0; o->nDivCor = 0; o->failed = 0;
    memset(o->EMrelErr, 0, sizeof(double) * o->MaxDivCor * o->IterPerDivCor);
    memset(o->divJ, 0, sizeof(double) * 2 * o->MaxDivCor);
    memset(o->DivCorIters, 0, sizeof(int) * o->MaxDivCor);
    int nonzero_source = (src != NULL);
    int nonzero_bc = (bc != NULL);
    if (nonzero_source) phi0 = xcalloc(nN, sizeof(cplx));
    if (trans) {
        if (!nonzero_source) {
            for (long i = 0; i < nE; i++) e[i] = 0.0;
            if (nonzero_bc)
                for (long i = 0; i < nE; i++) if (!orc_is_interior_edge(o, i)) e[i] = bc[i];
            free(b); free(temp);
            return 0;
        }
        for (long i = 0; i < nE; i++) b[i] = orc_is_interior_edge(o, i) ? src[i] : 0.0;
        for (long i = 0; i < nE; i++) temp[i] = b[i] / o->VE[i];
        div_plain(o, temp, phi0);
    } else {
        if (nonzero_bc) {
            for (long i = 0; i < nE; i++) temp[i] = orc_is_interior_edge(o, i) ? 0.0 : bc[i];
            multA_N(o, temp, 0, b);
            for (long i = 0; i < nE; i++) b[i] = -1.0 * b[i];
        }
        if (nonzero_source) {
            for (long i = 0; i < nE; i++) temp[i] = orc_is_interior_edge(o, i) ? src[i] : 0.0;
            div_plain(o, temp, phi0);
            for (long i = 0; i < nE; i++) temp[i] = o->VE[i] * temp[i];
            if (nonzero_bc) for (long i = 0; i < nE; i++) b[i] = temp[i] + b[i];
            else memcpy(b, temp, nE * sizeof(cplx));
        }
    }
    if (nonzero_source) for (long i = 0; i < nN; i++) phi0[i] = (1.0 / i_omega_mu) * phi0[i];
    /* first guess is zero on the boundary */
    for (long i = 0; i < nE; i++) if (!orc_is_interior_edge(o, i)) e[i] = 0.0;

    kss_t it = {0};
    it.tol = trans ? o->tolEMadj : (nonzero_bc ? o->tolEMfwd : o->tolEMadj);
    it.maxIt = o->IterPerDivCor;
    it.rerr = xcalloc(it.maxIt, sizeof(double));
    int converged = 0, failed = 0;
    if (nonzero_source) {
        o->nDivCor = 1;
        sdivcorr(o, e, phi0);
    }
    while (!converged && !failed) {
        it.niter = 0; it.failed = 0;
        memset(it.rerr, 0, sizeof(double) * it.maxIt);
        if (o->solver == ORC_QMR) qmr(o, b, e, &it);
        else if (o->solver == ORC_COCG) cocg(o, b, e, &it);
        else bicg(o, b, e, &it);
        converged = it.niter < it.maxIt;
        failed = failed || it.failed;
        for (int k = 0; k < it.niter; k++)
            if (o->nIterTotal + k < o->MaxDivCor * o->IterPerDivCor) o->EMrelErr[o->nIterTotal + k] = it.rerr[k];
        o->nIterTotal += it.niter;
        o->nDivCor++;
        if (o->nDivCor < o->MaxDivCor) sdivcorr(o, e, phi0);
        else failed = 1;
    }
    o->failed = failed;
    if (trans) {
        for (long i = 0; i < nE; i++) e[i] = o->VE[i] * e[i];
        cplx *tbc = xcalloc(nE, sizeof(cplx));
        adjt_bc(o, e, tbc);
        for (long i = 0; i < nE; i++)
            if (!orc_is_interior_edge(o, i)) e[i] = nonzero_bc ? (bc[i] - tbc[i]) : -tbc[i];
        free(tbc);
    } else {
        for (long i = 0; i < nE; i++)
            if (!orc_is_interior_edge(o, i)) e[i] = nonzero_bc ? bc[i] : 0.0;
    }
    free(b); free(temp); free(phi0); free(it.rerr);
    return converged ? 0 : 1;
}

/* Run one Krylov call (BICG or QMR per the control) on the interior system
 * A x = b with x the initial guess; returns niter, fills rerr. */
int orc_krylov(orc_t *o, const cplx *b, cplx *x, int maxit, double tol, double *rerr, int *failed)
{
    kss_t it = {0};
    it.maxIt = maxit; it.tol = tol;
    it.rerr = xcalloc(maxit, sizeof(double));
    if (o->solver == ORC_QMR) qmr(o, b, x, &it);
    else if (o->solver == ORC_COCG) cocg(o, b, x, &it);
    else bicg(o, b, x, &it);
    if (rerr) memcpy(rerr, it.rerr, sizeof(double) * maxit);
    if (failed) *failed = it.failed;
    free(it.rerr);
    return it.niter;
}

/* PmultT + EdgeToModelParam (f90/3D_MT/SolverSens.f90:63-116,
 * f90/3D_MT/modelParam/ModelMap.inc:302-374): gradient of a real functional
 * with respect to ln(sigma) of the earth cells, from the background fields e0
 * and adjoint fields eadj of npol polarisations (each a full edge vector).
 * dm has nx*ny*nzEarth entries. */
void orc_pmult_t(const orc_t *o, int npol, const cplx *e0, const cplx *eadj, const double *m0_earth, double *dm)
{
    long nE = o->nE;
    cplx minus_i_omega_mu = CMPLX(0.0, -ISIGN * MU_0 * o->omega);
    cplx *Ct = xcalloc(nE, sizeof(cplx));
    for (long i = 0; i < nE; i++) Ct[i] = e0[i] * eadj[i];
    for (int k = 1; k < npol; k++)
        for (long i = 0; i < nE; i++) Ct[i] = Ct[i] + e0[(size_t)k * nE + i] * eadj[(size_t)k * nE + i];
    for (long i = 0; i < nE; i++) Ct[i] = minus_i_omega_mu * Ct[i];
    double *temp = xcalloc(nE, sizeof(double)), *VEg = xcalloc(nE, sizeof(double));
    double *Ctemp = xcalloc(o->nC, sizeof(double));
    for (long i = 0; i < nE; i++) temp[i] = creal(Ct[i]);
    cell2edge(o, o->VC, VEg);
    for (long i = 0; i < nE; i++) temp[i] = temp[i] / VEg[i];
    edge2cell(o, temp, Ctemp);
    long off = (long)o->nx * o->ny * o->nzAir;
    long nEarth = (long)o->nx * o->ny * (o->nz - o->nzAir);
    for (long i = 0; i < nEarth; i++) dm[i] = (Ctemp[off + i] * o->VC[off + i]) * exp(m0_earth[i]);
    free(Ct); free(temp); free(VEg); free(Ctemp);
}

/* accessors for the Python wrapper */
long orc_nE(const orc_t *o) { return o->nE; }
long orc_nN(const orc_t *o) { return o->nN; }
void orc_get_VE(const orc_t *o, double *out) { memcpy(out, o->VE, sizeof(double) * o->nE); }
void orc_get_VN(const orc_t *o, double *out) { memcpy(out, o->VN, sizeof(double) * o->nN); }
void orc_get_sigE(const orc_t *o, double *out) { memcpy(out, o->sigE, sizeof(double) * o->nE); }
void orc_get_sigC(const orc_t *o, double *out) { memcpy(out, o->sigC, sizeof(double) * o->nC); }
void orc_get_divcorr_coef(const orc_t *o, double *db1, double *db2, double *c)
{
    memcpy(db1, o->db1, sizeof(double) * o->nE);
    memcpy(db2, o->db2, sizeof(double) * o->nE);
    memcpy(c, o->c, sizeof(double) * o->nN);
}
void orc_get_diag(const orc_t *o, int *nIterTotal, int *nDivCor, int *failed, double *EMrelErr, double *divJ,
                  int *DivCorIters)
{
    *nIterTotal = o->nIterTotal;
    *nDivCor = o->nDivCor;
    *failed = o->failed;
    if (EMrelErr) memcpy(EMrelErr, o->EMrelErr, sizeof(double) * o->MaxDivCor * o->IterPerDivCor);
    if (divJ) memcpy(divJ, o->divJ, sizeof(double) * 2 * o->MaxDivCor);
    if (DivCorIters) memcpy(DivCorIters, o->DivCorIters, sizeof(int) * o->MaxDivCor);
}
double orc_mu0(void) { return MU_0; }
double orc_sigma_air(void) { return SIGMA_AIR; }
