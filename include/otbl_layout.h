/*
 * otbl_layout.h -- header-only memory layouts shared by every side of the
 * C ABI: the packed coefficient buffer and the field arrays.
 *
 * Field layout (identical to the reference's single-rank plane arrays,
 * Fortran column-major, rhsp.F90:43-45):
 *   u-type fields (u, w, rhsupa, rhswpa):  complex*16 (0:nz2, ny+1, nx)
 *   v-type fields (v, p, rhsvpa):          complex*16 (0:nz2, ny,   nx)
 * seen from C as doubles with the real index kr = 0..nz1-1 fastest
 * (kr = 2k is Re of spanwise mode k, kr = 2k+1 its Im), then the wall-normal
 * row j = 1..jee, then the streamwise plane i = 1..nx:
 *   offset(kr, j, i) = ((i-1)*jee + (j-1))*nz1 + kr
 * with nz1 = 2*(nz/3) and nz2 = nz1/2-1 (mod.F90:27).
 *
 * Coefficient buffer: every array the substep reads from the reference's
 * module alloc_dns (mod.F90:96-184), packed one after the other in the order
 * of OTBL_COEF_LIST. Each array keeps its Fortran column-major shape, e.g.
 * inxu(3,nx) occupies 3*nx doubles with inxu(r,i) at [(i-1)*3 + (r-1)], and
 * arrays with lower bound 0 (y(0:ny+1), dy(0:ny), ...) start at index 0.
 * The first block (SCAL) holds the scalars listed in OTBL_S_*. The last five
 * arrays (fd_dvdy, fd_dx, fd_ix, fd_iy, fd_iyp, each (8, n)) are the compact
 * operators of the one-point statistics (coeft.f90:56-318); the substep does
 * not read them.
 */
#ifndef OTBL_LAYOUT_H
#define OTBL_LAYOUT_H

#include <stddef.h>

/* X(name, length) ; lengths use NX, NY, NZ2 */
#define OTBL_COEF_LIST(X)                                                     \
  X(SCAL, 64)                                                                 \
  X(Y, NY + 2) X(DY, NY + 1) X(IDY, NY + 1) X(IDYY, NY) X(DYMIN, NY)          \
  X(HY, NY + 1) X(XG, NX + 2) X(DX, NX + 1)                                   \
  X(KAZ, NZ2 + 1) X(KAZ2, NZ2 + 1) X(KVIS, NZ2 + 1)                           \
  X(KMOD, NX - 1) X(AYP, 3 * NY) X(VMAGIC, NX)                                \
  X(INXU, 3 * NX) X(INXV, 3 * NX) X(COFIUX, 2 * NX) X(COFIVX, 2 * NX)         \
  X(INBX, 16)                                                                 \
  X(DCXU, 3 * NX) X(DCXV, 3 * NX) X(COFCXU, 2 * NX) X(COFCXV, 2 * NX)         \
  X(DCBX, 20)                                                                 \
  X(VIXU, 3 * NX) X(VIXV, 3 * NX) X(COFVXU, 3 * NX) X(COFVXV, 3 * NX)         \
  X(COFVBX, 16)                                                               \
  X(INYU, 3 * NY) X(INYV, 3 * NY) X(COFIUY, 2 * NY) X(COFIVY, 2 * NY)         \
  X(INBY, 16)                                                                 \
  X(DCYU, 3 * (NY + 1)) X(DCYV, 3 * NY) X(COFCYU, 2 * NY) X(COFCYV, 2 * NY)   \
  X(DCBY, 16)                                                                 \
  X(VIYU, 3 * (NY + 1)) X(VIYV, 3 * NY) X(VYUI, 3 * (NY + 1)) X(VYVI, 3 * NY) \
  X(COFVYU, 3 * NY) X(COFVYV, 3 * NY) X(COFVBY, 16) X(CCON, 8)                \
  X(FD_DVDY, 8 * NY) X(FD_DX, 8 * NX) X(FD_IX, 8 * NX) X(FD_IY, 8 * NY)       \
  X(FD_IYP, 8 * NY)

/* scalar slots inside the SCAL block */
enum {
  OTBL_S_RE = 0,    /* Reynolds number re                                  */
  OTBL_S_REX,       /* rex = -1/re                (coeft.f90:480)          */
  OTBL_S_AX, OTBL_S_AY, OTBL_S_AZ, OTBL_S_CFL,
  OTBL_S_DX1,       /* dx(1)                                               */
  OTBL_S_IDX,       /* idx  = 1/dx(1)             (coeft.f90:420)          */
  OTBL_S_IDXX,      /* idxx = 1/dx(1)             (coeft.f90:423)          */
  OTBL_S_DXMIN,     /* dxmin*cfl/sqrt(3)          (coeft.f90:453)          */
  OTBL_S_DZMIN,     /* dzmin*cfl/pi               (coeft.f90:454)          */
  OTBL_S_DTRET,     /* viscous dt limit           (coeft.f90:443)          */
  OTBL_S_PI,
  OTBL_S_UINF,      /* Uinfinity = 1              (mod.F90:47)             */
  OTBL_S_RTHIN,     /* inlet Re_theta             (bl_1.F90:388)           */
  OTBL_S_DIN,       /* inlet delta99              (bl_1.F90:387)           */
  OTBL_S_YBLEND,    /* height replacing y(119) in genflu.F90:57            */
  OTBL_S_RKC = 20,  /* rkc(1:3)   (coeft.f90:494-496)                      */
  OTBL_S_RKD = 23,  /* rkd(1:3)   (coeft.f90:498-500)                      */
  OTBL_S_RKCV = 26, /* rkcv(1:3)  (coeft.f90:502-504)                      */
  OTBL_S_RKDV = 29, /* rkdv(1:3)  (coeft.f90:506-508)                      */
  OTBL_S_NX = 40, OTBL_S_NY, OTBL_S_NZ, OTBL_S_XOUT /* sizes, as doubles   */
};

enum {
#define OTBL_X_ENUM(name, len) OTBL_C_##name,
  OTBL_COEF_LIST(OTBL_X_ENUM)
#undef OTBL_X_ENUM
  OTBL_C_COUNT
};

typedef struct otbl_coef_offsets {
  size_t off[OTBL_C_COUNT + 1]; /* off[OTBL_C_COUNT] = total length */
} otbl_coef_offsets;

static inline void otbl_coef_layout(int nx, int ny, int nz,
                                    otbl_coef_offsets *o) {
  const long NX = nx, NY = ny, NZ2 = (2 * (nz / 3)) / 2 - 1;
  size_t cur = 0;
  int id = 0;
#define OTBL_X_OFF(name, len) \
  o->off[id++] = cur;         \
  cur += (size_t)(len);
  OTBL_COEF_LIST(OTBL_X_OFF)
#undef OTBL_X_OFF
  o->off[OTBL_C_COUNT] = cur;
  (void)NX; (void)NY; (void)NZ2;
}

/* number of doubles of one u-type / v-type field */
static inline size_t otbl_field_len(int nx, int ny, int nz, int utype) {
  const size_t nz1 = (size_t)(2 * (nz / 3));
  return (size_t)nx * (size_t)(utype ? ny + 1 : ny) * nz1;
}

#endif
