/*
 * CPU restatement of the reference per-patch Poisson-gravity path, generic in
 * the element type.  TEST INFRASTRUCTURE ONLY: the parity checker for the CUDA
 * library and the CPU baseline of the benchmark; never part of the product.
 *
 * Included twice by gpg_oracle.c with
 *   T      element type (float | double)
 *   SFX    name suffix  (f32 | f64)
 *   TABS   |x| for T    (fabsf | fabs)
 *
 * Every arithmetic expression keeps the operand order of the reference CPU
 * solver it follows, so that with gcc's baseline x86-64 code (no FMA) the
 * results are bit-identical to the reference compiled the same way.
 */

#define GPG_CAT2(a, b) a##_##b
#define GPG_CAT(a, b) GPG_CAT2(a, b)
#define FN(name) GPG_CAT(name, SFX)

/* Coarse -> fine interpolation of one patch into the solver cube.
 * cube is N^3 (N = 8+2g) and holds the fine cells [u, NI-u)^3 of the
 * reference's Pot_Array_Int (NI = 2*(POT_NXT-2), u = g%2).
 * CQUAD follows CPU_PoissonSolver_SOR.cpp:110-174 (13 slopes with weights
 * 1/8, 1/64, 1/512); QUAD follows CPU_PoissonSolver_SOR.cpp:177-203 (27-point
 * tensor product of Mm = {5,30,-3}/32, Mp = {-3,30,5}/32). */
static void FN(oracle_interp)(const T *cp, T *cube, int g, int int_scheme)
{
   const int pint = (g + 3) / 2, pn = 4 + 2 * pint, N = 8 + 2 * g, u = g % 2;
   const T c8 = (T)1.0 / (T)8.0, c64 = (T)1.0 / (T)64.0, c512 = (T)1.0 / (T)512.0;
   const T Mm[3] = {(T)(5.0 / 32.0), (T)(30.0 / 32.0), (T)(-3.0 / 32.0)};
   const T Mp[3] = {(T)(-3.0 / 32.0), (T)(30.0 / 32.0), (T)(5.0 / 32.0)};
#define CP(k, j, i) cp[((size_t)(k) * pn + (j)) * pn + (i)]

   for (int k = 1; k < pn - 1; k++)
   for (int j = 1; j < pn - 1; j++)
   for (int i = 1; i < pn - 1; i++) {
      T child[8];
      if (int_scheme == GPG_INT_CQUAD) {
         const int kp = k + 1, km = k - 1, jp = j + 1, jm = j - 1, ip = i + 1, im = i - 1;
         T s[13];
         s[0] = c8 * (CP(k, j, ip) - CP(k, j, im));
         s[1] = c8 * (CP(k, jp, i) - CP(k, jm, i));
         s[2] = c8 * (CP(kp, j, i) - CP(km, j, i));
         s[3] = c64 * (CP(km, j, ip) - CP(km, j, im));
         s[4] = c64 * (CP(km, jp, i) - CP(km, jm, i));
         s[5] = c64 * (CP(k, jm, ip) - CP(k, jm, im));
         s[6] = c64 * (CP(k, jp, ip) - CP(k, jp, im));
         s[7] = c64 * (CP(kp, j, ip) - CP(kp, j, im));
         s[8] = c64 * (CP(kp, jp, i) - CP(kp, jm, i));
         s[9] = c512 * (CP(km, jm, ip) - CP(km, jm, im));
         s[10] = c512 * (CP(km, jp, ip) - CP(km, jp, im));
         s[11] = c512 * (CP(kp, jm, ip) - CP(kp, jm, im));
         s[12] = c512 * (CP(kp, jp, ip) - CP(kp, jp, im));
         for (int c = 0; c < 8; c++) {
            /* child c: bit0 = +x half, bit1 = +y half, bit2 = +z half.  The
             * sign of each slope term is a product of the half-signs; the
             * terms are summed in slope order and the cell value added last. */
            const T sx = (c & 1) ? (T)1 : (T)-1, sy = (c & 2) ? (T)1 : (T)-1,
                    sz = (c & 4) ? (T)1 : (T)-1;
            const T sgn[13] = {sx, sy, sz, -sx * sz, -sy * sz, -sx * sy, sx * sy, sx * sz,
                               sy * sz, sx * sy * sz, -sx * sy * sz, -sx * sy * sz,
                               sx * sy * sz};
            T v = sgn[0] * s[0];
            for (int t = 1; t < 13; t++) v = v + sgn[t] * s[t];
            child[c] = v + CP(k, j, i);
         }
      } else {
         for (int c = 0; c < 8; c++) {
            const T *Wx = (c & 1) ? Mp : Mm, *Wy = (c & 2) ? Mp : Mm, *Wz = (c & 4) ? Mp : Mm;
            T v = (T)0.0;
            for (int dk = -1; dk <= 1; dk++)
            for (int dj = -1; dj <= 1; dj++)
            for (int di = -1; di <= 1; di++)
               v += CP(k + dk, j + dj, i + di) * Wz[dk + 1] * Wy[dj + 1] * Wx[di + 1];
            child[c] = v;
         }
      }
      for (int c = 0; c < 8; c++) {
         const int x = 2 * (i - 1) + (c & 1) - u, y = 2 * (j - 1) + ((c >> 1) & 1) - u,
                   z = 2 * (k - 1) + ((c >> 2) & 1) - u;
         if (x < 0 || y < 0 || z < 0 || x >= N || y >= N || z >= N) continue;
         cube[((size_t)z * N + y) * N + x] = child[c];
      }
   }
#undef CP
}

/* Red-black SOR of one patch (CPU_PoissonSolver_SOR.cpp:213-283).
 * Pass p updates interior cells (a,b,c) with (a+b+c)%2 == p in c, b, a order:
 *   R = phi(z+1)+phi(z-1)+phi(y+1)+phi(y-1)+phi(x+1)+phi(x-1) - 6 phi - Const rho
 *   phi += Omega/6 * R,   Total += |R|
 * accum_f64 selects a double accumulator for Total (the CUDA kernels' choice)
 * instead of the reference's `real` one.  Returns the sweep count. */
static int FN(oracle_sor_patch)(T *cube, const T *rho, int g, T Const, T Omega_6,
                                int min_iter, int max_iter, int stop_mode, double tol_abs,
                                int accum_f64, double *resid_out)
{
   const int N = 8 + 2 * g, M = N - 2;
   T total_old_r = (T)3.40282347e+38F; /* __FLT_MAX__ */
   double total_old_d = 3.40282347e+38F;
   double last = 0.0;
   int iter;
#define PH(z, y, x) cube[((size_t)(z) * N + (y)) * N + (x)]
   for (iter = 0; iter < max_iter; iter++) {
      T total_r = (T)0.0;
      double total_d = 0.0;
      for (int pass = 0; pass < 2; pass++)
      for (int c = 0; c < M; c++)
      for (int b = 0; b < M; b++)
      for (int a = (pass + b + c) & 1; a < M; a += 2) {
         const int z = c + 1, y = b + 1, x = a + 1;
         const T R = (PH(z + 1, y, x) + PH(z - 1, y, x) + PH(z, y + 1, x) + PH(z, y - 1, x) +
                      PH(z, y, x + 1) + PH(z, y, x - 1) - (T)6.0 * PH(z, y, x) -
                      Const * rho[((size_t)c * M + b) * M + a]);
         PH(z, y, x) += Omega_6 * R;
         if (accum_f64) total_d += (double)TABS(R);
         else           total_r += TABS(R);
      }
      last = accum_f64 ? total_d : (double)total_r;
      if (stop_mode == GPG_STOP_REFERENCE) {
         const int grew = accum_f64 ? (total_d > total_old_d) : (total_r > total_old_r);
         if (iter + 1 >= min_iter && grew) { iter++; break; }
      } else {
         if (iter + 1 >= min_iter && last <= tol_abs) { iter++; break; }
      }
      total_old_r = total_r;
      total_old_d = total_d;
   }
#undef PH
   if (resid_out) *resid_out = last;
   return iter;
}

/* ---- multigrid helpers, CPU_PoissonSolver_MG.cpp:392-684 ---------------- */

/* Gauss-Seidel red-black smoothing (CPU_PoissonSolver_MG.cpp:392-441):
 * pass 0 updates cells with (i+j+k) odd, pass 1 the rest. */
static void FN(mg_smooth)(T *sol, const T *rhs, T dh, int n)
{
   const T dh2 = dh * dh, one_six = (T)1.0 / (T)6.0;
#define S(k, j, i) sol[((size_t)(k) * n + (j)) * n + (i)]
   for (int pass = 0; pass < 2; pass++)
   for (int k = 1; k < n - 1; k++)
   for (int j = 1; j < n - 1; j++)
   for (int i = 2 - ((1 + k + j + pass) & 1); i < n - 1; i += 2)
      S(k, j, i) = one_six * (S(k + 1, j, i) + S(k - 1, j, i) + S(k, j + 1, i) + S(k, j - 1, i) +
                              S(k, j, i + 1) + S(k, j, i - 1) -
                              dh2 * rhs[((size_t)k * n + j) * n + i]);
#undef S
}

/* Negative defect -(lap(sol) - rhs) on interior cells (CPU_PoissonSolver_MG.cpp:460-495). */
static void FN(mg_defect)(const T *sol, const T *rhs, T *def, T dh, int n)
{
   const T m_dh2 = (T)-1.0 / (dh * dh);
#define S(k, j, i) sol[((size_t)(k) * n + (j)) * n + (i)]
   for (int k = 1; k < n - 1; k++)
   for (int j = 1; j < n - 1; j++)
   for (int i = 1; i < n - 1; i++) {
      const size_t id = ((size_t)k * n + j) * n + i;
      def[id] = m_dh2 * (S(k + 1, j, i) + S(k - 1, j, i) + S(k, j + 1, i) + S(k, j - 1, i) +
                         S(k, j, i + 1) + S(k, j, i - 1) - (T)6.0 * S(k, j, i)) + rhs[id];
   }
#undef S
}

/* L1 error estimate dh^2 sum|def| / sum|sol| (CPU_PoissonSolver_MG.cpp:497-512);
 * with accum_f64 the sums and the ratio are formed in double. */
static double FN(mg_error)(const T *sol, const T *def, T dh, int n, int accum_f64)
{
   T sd = (T)0.0, ss = (T)0.0;
   double sdd = 0.0, ssd = 0.0;
   for (int k = 1; k < n - 1; k++)
   for (int j = 1; j < n - 1; j++)
   for (int i = 1; i < n - 1; i++) {
      const size_t id = ((size_t)k * n + j) * n + i;
      if (accum_f64) { sdd += (double)TABS(def[id]); ssd += (double)TABS(sol[id]); }
      else           { sd += TABS(def[id]); ss += TABS(sol[id]); }
   }
   if (accum_f64) return ((double)(dh * dh) * sdd) / ssd;
   return (double)(dh * dh * sd / ss);
}

/* Full-weighting style 27-point restriction of vertex-centred data
 * (CPU_PoissonSolver_MG.cpp:533-616); boundary values of cdata untouched. */
static void FN(mg_restrict)(const T *f, T *cdat, int nf, int nc)
{
   const T ratio = (T)(nf - 1) / (T)(nc - 1);
#define F(k, j, i) f[((size_t)(k) * nf + (j)) * nf + (i)]
   for (int k = 1; k < nc - 1; k++) {
      const T z = k * ratio;
      const int kk = (int)(z + (T)0.5);
      T cz[3];
      cz[0] = (T)0.5 * (kk + (T)0.5 - z);
      cz[2] = (T)0.5 - cz[0];
      cz[1] = (T)0.5;
      for (int j = 1; j < nc - 1; j++) {
         const T y = j * ratio;
         const int jj = (int)(y + (T)0.5);
         T cy[3];
         cy[0] = (T)0.5 * (jj + (T)0.5 - y);
         cy[2] = (T)0.5 - cy[0];
         cy[1] = (T)0.5;
         for (int i = 1; i < nc - 1; i++) {
            const T x = i * ratio;
            const int ii = (int)(x + (T)0.5);
            T cx[3];
            cx[0] = (T)0.5 * (ii + (T)0.5 - x);
            cx[2] = (T)0.5 - cx[0];
            cx[1] = (T)0.5;
            T v = cz[0] * cy[0] * cx[0] * F(kk - 1, jj - 1, ii - 1);
            for (int t = 1; t < 27; t++) {
               const int dz = t / 9, dy = (t / 3) % 3, dx = t % 3;
               v = v + cz[dz] * cy[dy] * cx[dx] * F(kk - 1 + dz, jj - 1 + dy, ii - 1 + dx);
            }
            cdat[((size_t)k * nc + j) * nc + i] = v;
         }
      }
   }
#undef F
}

/* Trilinear prolongation added to interior fine cells
 * (CPU_PoissonSolver_MG.cpp:635-684).  The eight corner terms are summed in
 * the reference's order: 000, 001, 010, 100, 011, 110, 101, 111 (z,y,x bits). */
static void FN(mg_prolongate)(const T *cdat, T *f, int nc, int nf)
{
   static const int order[8][3] = {{0, 0, 0}, {0, 0, 1}, {0, 1, 0}, {1, 0, 0},
                                   {0, 1, 1}, {1, 1, 0}, {1, 0, 1}, {1, 1, 1}};
   const T ratio = (T)(nc - 1) / (T)(nf - 1);
#define C(k, j, i) cdat[((size_t)(k) * nc + (j)) * nc + (i)]
   for (int k = 1; k < nf - 1; k++) {
      const T z = k * ratio;
      const int kk = (int)z;
      T cz[2];
      cz[0] = (kk + 1) - z;
      cz[1] = (T)1.0 - cz[0];
      for (int j = 1; j < nf - 1; j++) {
         const T y = j * ratio;
         const int jj = (int)y;
         T cy[2];
         cy[0] = (jj + 1) - y;
         cy[1] = (T)1.0 - cy[0];
         for (int i = 1; i < nf - 1; i++) {
            const T x = i * ratio;
            const int ii = (int)x;
            T cx[2];
            cx[0] = (ii + 1) - x;
            cx[1] = (T)1.0 - cx[0];
            T v = cz[0] * cy[0] * cx[0] * C(kk, jj, ii);
            for (int t = 1; t < 8; t++) {
               const int oz = order[t][0], oy = order[t][1], ox = order[t][2];
               v = v + cz[oz] * cy[oy] * cx[ox] * C(kk + oz, jj + oy, ii + ox);
            }
            f[((size_t)k * nf + j) * nf + i] += v;
         }
      }
   }
#undef C
}

/* Multigrid V-cycles of one patch (CPU_PoissonSolver_MG.cpp:62-87, 256-325).
 * lv arrays: sol/rhs/def per level, n[lv] cells per side.  Returns V-cycles. */
static int FN(oracle_mg_patch)(T *sol0, const T *rho, int g, T dh_min, T poi_coeff, int max_iter,
                               int npre, int npost, T tol, int accum_f64, double *err_out,
                               T **sol, T **rhs, T **def, const int *n, const T *dhl, int bottom,
                               int nbottom)
{
   const int M = 6 + 2 * g, N0 = n[0];
   (void)sol0;
   for (int k = 0; k < M; k++)
   for (int j = 0; j < M; j++)
   for (int i = 0; i < M; i++)
      rhs[0][((size_t)(k + 1) * N0 + (j + 1)) * N0 + (i + 1)] =
         poi_coeff * rho[((size_t)k * M + j) * M + i];

   int iter = 0;
   T err_r = (T)3.40282347e+38F;
   double err_d = 3.40282347e+38F;
   while (iter < max_iter && (accum_f64 ? (err_d > (double)tol) : (err_r > tol))) {
      for (int lv = 0; lv < bottom; lv++) {
         for (int s = 0; s < npre; s++) FN(mg_smooth)(sol[lv], rhs[lv], dhl[lv], n[lv]);
         FN(mg_defect)(sol[lv], rhs[lv], def[lv], dhl[lv], n[lv]);
         FN(mg_restrict)(def[lv], rhs[lv + 1], n[lv], n[lv + 1]);
         const size_t cnt = (size_t)n[lv + 1] * n[lv + 1] * n[lv + 1];
         for (size_t t = 0; t < cnt; t++) sol[lv + 1][t] = (T)0.0;
      }
      for (int s = 0; s < nbottom; s++) FN(mg_smooth)(sol[bottom], rhs[bottom], dhl[bottom], n[bottom]);
      for (int lv = bottom - 1; lv >= 0; lv--) {
         FN(mg_prolongate)(sol[lv + 1], sol[lv], n[lv + 1], n[lv]);
         for (int s = 0; s < npost; s++) FN(mg_smooth)(sol[lv], rhs[lv], dhl[lv], n[lv]);
      }
      FN(mg_defect)(sol[0], rhs[0], def[0], dhl[0], n[0]);
      const double e = FN(mg_error)(sol[0], def[0], dhl[0], n[0], accum_f64);
      if (accum_f64) err_d = e;
      else {
         /* recompute in T exactly as the reference does */
         err_r = (T)e;
      }
      iter++;
   }
   if (err_out) *err_out = accum_f64 ? err_d : (double)err_r;
   return iter;
}

/* Gravity update of one patch (CPU_GravitySolver.cpp:17-81). */
static void FN(oracle_gravity_patch)(T *flu, const T *pot, int G, T gra_const, int p5)
{
   const int GN = 8 + 2 * G, PS = 8;
   const T c8 = (T)8.0;
#define P(k, j, i) pot[((size_t)(k) * GN + (j)) * GN + (i)]
   for (int k = G; k < GN - G; k++)
   for (int j = G; j < GN - G; j++)
   for (int i = G; i < GN - G; i++) {
      T acc[3];
      if (G == 2 && p5) {
         acc[0] = gra_const * (-P(k, j, i + 2) + P(k, j, i - 2) + c8 * P(k, j, i + 1) - c8 * P(k, j, i - 1));
         acc[1] = gra_const * (-P(k, j + 2, i) + P(k, j - 2, i) + c8 * P(k, j + 1, i) - c8 * P(k, j - 1, i));
         acc[2] = gra_const * (-P(k + 2, j, i) + P(k - 2, j, i) + c8 * P(k + 1, j, i) - c8 * P(k - 1, j, i));
      } else {
         acc[0] = gra_const * (P(k, j, i + 1) - P(k, j, i - 1));
         acc[1] = gra_const * (P(k, j + 1, i) - P(k, j - 1, i));
         acc[2] = gra_const * (P(k + 1, j, i) - P(k - 1, j, i));
      }
      const size_t c = ((size_t)(k - G) * PS + (j - G)) * PS + (i - G), vs = (size_t)PS * PS * PS;
      const T rho = flu[c], temp = (T)0.5 / rho;
      T px = flu[vs + c], py = flu[2 * vs + c], pz = flu[3 * vs + c];
      const T eint = flu[4 * vs + c] - temp * (px * px + py * py + pz * pz);
      px -= rho * acc[0];
      py -= rho * acc[1];
      pz -= rho * acc[2];
      flu[vs + c] = px;
      flu[2 * vs + c] = py;
      flu[3 * vs + c] = pz;
      flu[4 * vs + c] = eint + temp * (px * px + py * py + pz * pz);
   }
#undef P
}

/* Batched driver with the argument list of CPU_PoissonGravitySolver
 * (CPU_PoissonGravitySolver.cpp:133-168): Poisson (SOR or MG) then gravity. */
int FN(oracle_poisson_gravity)(const gpg_params *prm, int npatch, const T *rho_all,
                               const T *pin_all, T *pout_all, T *flu_all, const T *guess_all,
                               int accum_f64, int nthreads, int32_t *iters, double *resid)
{
   const int g = prm->ghost, G = prm->gra_ghost;
   if (g < 1 || g > 5 || G < 0 || G > 2 || G > g || npatch < 0) return GPG_ERR_INVALID;
   if (prm->poisson && prm->int_scheme != GPG_INT_CQUAD && prm->int_scheme != GPG_INT_QUAD)
      return GPG_ERR_INVALID;
   if (prm->p5_gradient && G != 2 && prm->gra_acc) return GPG_ERR_INVALID;
   const int N = 8 + 2 * g, M = N - 2, pint = (g + 3) / 2, pn = 4 + 2 * pint, GN = 8 + 2 * G;
   const size_t sr = (size_t)M * M * M, sp = (size_t)pn * pn * pn, so = (size_t)GN * GN * GN,
                sf = 5 * 512, sc = (size_t)N * N * N;
   const T dt = (T)prm->dt, dh = (T)prm->dh, poi = (T)prm->poi_coeff;
   const int shift = g - G;

#ifdef _OPENMP
   if (nthreads > 0) omp_set_num_threads(nthreads);
#else
   (void)nthreads;
#endif

   if (prm->poisson && prm->scheme == GPG_SOR) {
      const T Const = poi * dh * dh, Omega = (T)prm->sor_omega, Omega_6 = Omega / (T)6.0;
#pragma omp parallel
      {
         T *cube = (T *)malloc(sc * sizeof(T));
#pragma omp for schedule(dynamic, 4)
         for (int P = 0; P < npatch; P++) {
            const T *rho = rho_all + (size_t)P * sr;
            FN(oracle_interp)(pin_all + (size_t)P * sp, cube, g, prm->int_scheme);
            double pot_sum = 0.0;   /* GPG_STOP_POT_TOLERANCE scale, before the guess */
            if (prm->stop_mode == GPG_STOP_POT_TOLERANCE)
               for (int c = 0; c < M; c++)
               for (int b = 0; b < M; b++)
               for (int a = 0; a < M; a++)
                  pot_sum += (double)TABS(cube[((size_t)(c + 1) * N + (b + 1)) * N + (a + 1)]);
            if (prm->init_mode != GPG_INIT_INTERP)
               for (int c = 0; c < M; c++)
               for (int b = 0; b < M; b++)
               for (int a = 0; a < M; a++)
                  cube[((size_t)(c + 1) * N + (b + 1)) * N + (a + 1)] =
                     prm->init_mode == GPG_INIT_GUESS
                        ? guess_all[(size_t)P * sr + ((size_t)c * M + b) * M + a] : (T)0.0;
            double tol_abs = prm->sor_tolerance;  /* GPG_STOP_ABS_TOLERANCE */
            if (prm->stop_mode == GPG_STOP_TOLERANCE) {
               double s = 0.0;
               for (size_t t = 0; t < sr; t++) s += (double)TABS(Const * rho[t]);
               tol_abs = prm->sor_tolerance * s;
            } else if (prm->stop_mode == GPG_STOP_POT_TOLERANCE) {
               tol_abs = prm->sor_tolerance * pot_sum;
            }
            double r = 0.0;
            const int it = FN(oracle_sor_patch)(cube, rho, g, Const, Omega_6, prm->sor_min_iter,
                                                prm->sor_max_iter, prm->stop_mode, tol_abs,
                                                accum_f64, &r);
            if (iters) iters[P] = it;
            if (resid) resid[P] = r;
            T *out = pout_all + (size_t)P * so;
            for (int k = 0; k < GN; k++)
            for (int j = 0; j < GN; j++)
            for (int i = 0; i < GN; i++)
               out[((size_t)k * GN + j) * GN + i] =
                  cube[((size_t)(k + shift) * N + (j + shift)) * N + (i + shift)];
         }
         free(cube);
      }
   } else if (prm->poisson && prm->scheme == GPG_MG) {
      int n[10], bottom = 0;
      T dhl[10];
      n[0] = N;
      dhl[0] = dh;
      while ((n[bottom] + 1) / 2 >= 3 && bottom + 1 < 10) {
         bottom++;
         n[bottom] = (n[bottom - 1] + 1) / 2;
         dhl[bottom] = dh * (T)(n[0] - 1) / (T)(n[bottom] - 1);
      }
      int nbottom;
      if (n[bottom] == 3) nbottom = 1;
      else if (n[bottom] == 4) nbottom = 7;
      else return GPG_ERR_UNSUPPORTED;
#pragma omp parallel
      {
         T *sol[10], *rhs[10], *def[10];
         for (int lv = 0; lv <= bottom; lv++) {
            const size_t c = (size_t)n[lv] * n[lv] * n[lv];
            sol[lv] = (T *)malloc(c * sizeof(T));
            rhs[lv] = (T *)calloc(c, sizeof(T));
            def[lv] = (T *)calloc(c, sizeof(T));
         }
#pragma omp for schedule(dynamic, 4)
         for (int P = 0; P < npatch; P++) {
            FN(oracle_interp)(pin_all + (size_t)P * sp, sol[0], g, prm->int_scheme);
            double e = 0.0;
            const int it = FN(oracle_mg_patch)(sol[0], rho_all + (size_t)P * sr, g, dh, poi,
                                               prm->mg_max_iter, prm->mg_npre_smooth,
                                               prm->mg_npost_smooth, (T)prm->mg_tolerated_error,
                                               accum_f64, &e, sol, rhs, def, n, dhl, bottom,
                                               nbottom);
            if (iters) iters[P] = it;
            if (resid) resid[P] = e;
            T *out = pout_all + (size_t)P * so;
            for (int k = 0; k < GN; k++)
            for (int j = 0; j < GN; j++)
            for (int i = 0; i < GN; i++)
               out[((size_t)k * GN + j) * GN + i] =
                  sol[0][((size_t)(k + shift) * N + (j + shift)) * N + (i + shift)];
         }
         for (int lv = 0; lv <= bottom; lv++) { free(sol[lv]); free(rhs[lv]); free(def[lv]); }
      }
   } else if (prm->poisson) {
      return GPG_ERR_INVALID;
   }

   if (prm->gra_acc) {
      const T gra_const = prm->p5_gradient ? (T)((double)dt / (12.0 * (double)dh))
                                           : (T)((double)dt / (2.0 * (double)dh));
#pragma omp parallel for schedule(static)
      for (int P = 0; P < npatch; P++)
         FN(oracle_gravity_patch)(flu_all + (size_t)P * sf, pout_all + (size_t)P * so, G, gra_const,
                                  prm->p5_gradient);
   }
   return GPG_OK;
}

#undef FN
#undef GPG_CAT
#undef GPG_CAT2
