/*
 * gpg_cuapi.h -- the reference testbed's GPU call surface, unchanged, on top of
 * libgpg (include/gpg.h).  C++ only.
 *
 * These are exactly the prototypes of Header/Prototype.h:15-35 of
 * gamer-project/gpu_testbed_poisson-gravity.  Like the reference, the array
 * types depend on compile-time macros, so the implementation
 * (gpu_testbed_poisson-gravity_b200/csrc/cuapi/cuapi_compat.cpp) is compiled
 * with the caller's own flags:
 *   -DPATCH_SIZE=8 -DPOT_GHOST_SIZE=<1..5> -DGRA_GHOST_SIZE=<0..2>
 *   -DPOT_SCHEME=SOR|MG (SOR=1, MG=2) [-DFLOAT8]
 * and linked with libgpg.so.  A caller that already includes the reference's
 * Header/GAMER.h gets the same declarations from there; this header serves
 * callers (and the shim itself) that do not.
 *
 * Error behaviour matches the reference: a failure prints a message to stderr
 * and ends the process with exit(-1) (Header/CUAPI.h:10-21, Prototype.h:44).
 */
#ifndef GPG_CUAPI_H
#define GPG_CUAPI_H

#ifndef __cplusplus
#error "gpg_cuapi.h declares C++ functions"
#endif

#if !defined(PATCH_SIZE) || !defined(POT_GHOST_SIZE) || !defined(GRA_GHOST_SIZE) || !defined(POT_SCHEME)
#error "define PATCH_SIZE, POT_GHOST_SIZE, GRA_GHOST_SIZE and POT_SCHEME as for the caller"
#endif

#ifndef GPG_CUAPI_NO_TYPES
/* `real` and the interpolation-scheme enum, as in Header/Macro.h:35-39 and
 * Header/Typedef.h:7-8 (the enum's name is part of the C++ linkage names). */
#ifdef FLOAT8
typedef double real;
#else
typedef float real;
#endif
enum IntScheme_t { INT_DEFAULT = -1, INT_NONE = 0, INT_MINMOD3D = 1, INT_MINMOD1D = 2, INT_VANLEER = 3,
                   INT_CQUAD = 4, INT_QUAD = 5, INT_CQUAR = 6, INT_QUAR = 7 };
#endif

/* Derived sizes, Header/Macro.h:53-61. */
#ifndef RHO_NXT
#define GPG_CUAPI_POT_INT ((POT_GHOST_SIZE == 0) ? 0 : (POT_GHOST_SIZE + 3) / 2)
#define POT_NXT (PATCH_SIZE / 2 + 2 * GPG_CUAPI_POT_INT)
#define RHO_NXT (PATCH_SIZE + 2 * (POT_GHOST_SIZE - 1))
#define GRA_NXT (PATCH_SIZE + 2 * GRA_GHOST_SIZE)
#endif
#ifndef NCOMP
#define NCOMP 5
#endif

/* Header/Prototype.h:15 */
void CUAPI_Set_Diagnose_Device(int &FLU_GPU_NPGroup, int &GPU_NStream, const int InputID);
/* Header/Prototype.h:16-20 */
void CUAPI_MemAllocate_PoissonGravity(const int Pot_NPatchGroup,
                                      real (**Rho_Array_P)[RHO_NXT][RHO_NXT][RHO_NXT],
                                      real (**Pot_Array_P_In)[POT_NXT][POT_NXT][POT_NXT],
                                      real (**Pot_Array_P_Out)[GRA_NXT][GRA_NXT][GRA_NXT],
                                      real (**Flu_Array_G)[NCOMP][PATCH_SIZE][PATCH_SIZE][PATCH_SIZE]);
/* Header/Prototype.h:21-24 */
void CUAPI_MemFree_PoissonGravity(real (**Rho_Array_P)[RHO_NXT][RHO_NXT][RHO_NXT],
                                  real (**Pot_Array_P_In)[POT_NXT][POT_NXT][POT_NXT],
                                  real (**Pot_Array_P_Out)[GRA_NXT][GRA_NXT][GRA_NXT],
                                  real (**Flu_Array_G)[NCOMP][PATCH_SIZE][PATCH_SIZE][PATCH_SIZE]);
/* Header/Prototype.h:25-34 (asynchronous: call CUAPI_Synchronize before reading outputs) */
void CUAPI_Asyn_PoissonGravitySolver(const real h_Rho_Array[][RHO_NXT][RHO_NXT][RHO_NXT],
                                     real h_Pot_Array_In[][POT_NXT][POT_NXT][POT_NXT],
                                     real h_Pot_Array_Out[][GRA_NXT][GRA_NXT][GRA_NXT],
                                     real h_Flu_Array[][5][PATCH_SIZE][PATCH_SIZE][PATCH_SIZE],
                                     const int NPatchGroup, const real dt, const real dh,
                                     const int SOR_Min_Iter, const int SOR_Max_Iter, const real SOR_Omega,
                                     const int MG_Max_Iter, const int MG_NPre_Smooth,
                                     const int MG_NPost_Smooth, const real MG_Tolerated_Error,
                                     const real Poi_Coeff, const IntScheme_t IntScheme,
                                     const bool P5_Gradient, const bool Poisson, const bool GraAcc,
                                     const int GPU_NStream);
/* Header/Prototype.h:35 */
void CUAPI_Synchronize();

#endif /* GPG_CUAPI_H */
