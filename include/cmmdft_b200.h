/* cmmdft_b200 — C ABI of the B200 (sm_100a) classical-DFT grid solve.
 *
 * Every entry point takes plain pointers and sizes.  Pointers named d_* are
 * CUDA device pointers (FP64 unless stated); `stream` is a cudaStream_t
 * passed as void*.  All work is stream-ordered; nothing synchronises unless
 * the function says so.  Every function returns a cmm_status (0 = success).
 *
 * Data layout (one "shape group" of `batch` instances on an N1 x N2 x N3
 * grid, C order, x slowest as in the reference's Grid):
 *   real field  : double [batch][N1][N2][N3]
 *   spectrum    : double2 [batch][N1][N2][H3], H3 = N3/2 + 1, the 3D half
 *                 spectrum of a real field, x frequencies in natural order,
 *                 y and z frequencies in the plan's digit-reversed order.
 *                 Use cmm_spectrum_index() to map positions to frequencies.
 *   yz-spectrum : the same array shape with x still in real space and only
 *                 y, z transformed (the x transform lives inside the column
 *                 passes).  The functional pipeline and the solver plane
 *                 passes exchange densities and C1 in this layout.
 *
 * The reference (CmmDFT) is pure Python/numpy; it has no FFI.  Each entry
 * point below names the reference function whose arithmetic it replaces
 * (paths inside the reference project).
 */
#ifndef CMMDFT_B200_H
#define CMMDFT_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum cmm_status {
  CMM_OK = 0,
  CMM_ERR_ARG = 1,          /* bad argument (null pointer, negative size) */
  CMM_ERR_SHAPE = 2,        /* grid shape not supported by this build     */
  CMM_ERR_CUDA = 3,         /* a CUDA runtime call failed                 */
  CMM_ERR_SMEM = 4,         /* plane or tile does not fit in shared memory */
  CMM_ERR_NOMEM = 5,        /* allocation of plan tables failed           */
  CMM_ERR_WORKSPACE = 6,    /* caller workspace too small                 */
  CMM_ERR_UNSUPPORTED = 7   /* option not implemented                     */
} cmm_status;

/* Per-instance reduction slots written by the kernels (cmm_stats_finalize). */
enum {
  CMM_STAT_N = 0,        /* sum rho                                   */
  CMM_STAT_IUE = 1,      /* sum |rho - rho_ref|                       */
  CMM_STAT_NONFIN = 2,   /* count of non-finite rho                   */
  CMM_STAT_FID = 3,      /* sum rho_reg (ln(L^3 rho_reg) - 1)         */
  CMM_STAT_FEXT = 4,     /* sum rho V                                 */
  CMM_STAT_RES2 = 5,     /* sum (G - rho)^2                           */
  CMM_STAT_PHI = 6,      /* sum Phi (hard-sphere free-energy density) */
  CMM_STAT_MFA = 7,      /* Parseval sum for the MFA energy           */
  CMM_STAT_N3MAX = 8,    /* max n3 (unclipped)                        */
  CMM_STAT_GNONFIN = 9,  /* count of non-finite G                     */
  CMM_STAT_GRAM0 = 10,   /* sum r_new r_j, j = 0..CMM_MAX_HIST-1      */
  CMM_STAT_WDA = 18,     /* sum f_EOS(wd) (WDA free-energy density)   */
  CMM_STAT_DER = 19,     /* sum (rho beta dOmega / (a_tol + r_tol rho))^2 over rho != 0 */
  CMM_NSTAT = 20
};
#define CMM_MAX_HIST 8

/* Sums of the hybrid line search (cmm_ls_*), per instance [CMM_NLS]; the
 * trial densities are rho + alpha_i r, alpha_i = coef_i * alpha_max. */
enum {
  CMM_LS_MFA_RR = 0,    /* sum_k wt |r_k|^2 Re K (as CMM_STAT_MFA, for r)        */
  CMM_LS_MFA_XR = 1,    /* sum_k wt Re(conj(rho_k) r_k) Re K                      */
  CMM_LS_N3MAX_G = 2,   /* max over the grid of n3(rho) + n3(r) (= max n3 of G)   */
  CMM_LS_SUM_R = 3,     /* sum r                                                  */
  CMM_LS_SUM_RV = 4,    /* sum r V                                                */
  CMM_LS_FID = 5,       /* 5..7:  sum x (ln(L^3 x) - 1), x = rho + alpha_i r clipped as _clip_density */
  CMM_LS_PHI = 8,       /* 8..10: sum Phi(n(rho) + alpha_i n(r))                  */
  CMM_LS_WDA = 11,      /* 11..13: sum f_EOS(wd(rho) + alpha_i wd(r))             */
  CMM_NLS = 16
};

/* Hard-sphere functional versions (cmmdft/functionals.py:373-377): a base
 * (FMT, MFMT, WBII) with the 'a' (CMM_ANTISYM) and 't' (CMM_TENSOR, the six
 * tensor weighted densities of functionals.py:457-487, 534-552) options.
 * CMM_NOHS drops the hard-sphere term (the MFA convolution alone);
 * CMM_WDA adds the WDA correlation part described by a cmm_wda_eos. */
enum { CMM_FMT = 0, CMM_MFMT = 1, CMM_WBII = 2, CMM_ANTISYM = 8, CMM_NOHS = 16, CMM_WDA = 32, CMM_TENSOR = 64 };

/* WDA correlation part (WDAVFunctional with SumOfEOS([MBWR, CS, MFA],
 * factors), cmmdft/functionals.py:339-362, 1116-1184; cmmdft/eos.py).
 * Weight: 3 (sin x - x cos x) / x^3 sigma_L at x = |k| D.  The MBWR
 * coefficients a[8], b[6] are those at the solve temperature. */
typedef struct cmm_wda_eos {
  double D;                 /* weight diameter (2 Rhs); D < 0: the LDA part (LDAFunctional,
                               cmmdft/functionals.py:1085-1114), weight 1: the EOS at the density itself */
  double sigma3, epsilon, gamma;   /* MBWR: sigma**3 (as the reference forms it), epsilon, gamma */
  double a[8], b[6];
  double eta, kT;           /* Carnahan-Starling: 4 pi R^3 / 3, k_B T */
  double a_mfa;             /* mean-field EOS a */
  double factors[3];        /* SumOfEOS factors of MBWR, CS, MFA */
} cmm_wda_eos;

/* Mix-kernel clip modes. */
enum {
  CMM_CLIP_NONE = 0,
  CMM_CLIP_PICARD = 1,     /* rho < 1e-10 angstrom^-3 -> 0   (solver.py:398)      */
  CMM_CLIP_DENSITY = 2     /* rho < 1e-12 -> 1e-30          (solver.py:146-148)   */
};

typedef struct cmm_grid cmm_grid;

int cmm_version(void);
const char* cmm_status_string(int status);

/* Grid plan: twiddle tables, digit-reversal position tables and the k-space
 * tables of a periodic N1 x N2 x N3 grid (any sizes up to 1024; prime
 * factors > 16 run as Rader or direct-DFT stages; odd N3 as a full-length z
 * transform with the stored z frequencies in natural order) spanning the cell `rvecs` (3x3,
 * rows are cell vectors, bohr).  Replaces the k-grid, scalprod and Lanczos
 * tables of Grid.__init__ (cmmdft/system.py:232-295).  Allocates the plan's
 * device tables (the only persistent device memory this library owns). */
int cmm_grid_create(int n1, int n2, int n3, const double* rvecs, cmm_grid** out);
int cmm_grid_destroy(cmm_grid* grid);
/* Plane passes: a grid whose y-z plane of all fields fits in one SM's
 * shared memory runs the fused plane kernels (y and z transforms and the
 * pointwise step in one pass); larger planes, and the tensor variants, run
 * the staged form (a y pass over HBM, then z rows with the pointwise step).
 * mode 0 chooses by size (default), 1 always stages (tests, tuning), 2
 * chooses by size but runs the fused functional plane pass in one CTA per
 * plane instead of the default CTA pair (a 2-CTA cluster holding half of
 * the plane's fields each, two pairs per SM pair; bit-identical results).
 * Grids with odd N3 or a prime factor > 16 on the y or z axis always stage.
 * In the staged form cmm_residual_step and cmm_irfft_yz, whose spectrum
 * input is read-only, take a stream-ordered temporary of one spectrum per
 * instance (cudaMallocAsync / cudaFreeAsync on the call's stream). */
int cmm_grid_set_staging(cmm_grid* grid, int mode);
/* FFT schedules.  A plan's schedule fixes, per axis, the order of the
 * radix stages (CMM_ORDER_*), the form of the plane passes and the column
 * tile; all schedules give the same transforms up to rounding.  The
 * default (cmm_grid_create) is CMM_ORDER_DEFAULT everywhere, plane passes
 * by size, column tiles by size.  sched[5] = {x order, y order, z order
 * (-1: default), plane passes (-1 or 0: by size, 1: staged, 2: by size with
 * the one-CTA functional plane pass), column tile
 * width of the run-time-length column kernels (0: by size, else 1..16, a
 * power of two)}.  A non-default radix order runs the run-time-length
 * kernels on every axis (the compile-time ones for 32 and 64 points fix
 * their own order).  Used by the schedule autotuner
 * (cmmdft_b200/autotune.py), which times the candidates on the device. */
enum { CMM_ORDER_DEFAULT = 0,   /* 8s, 4s, 2s, then odd primes ascending        */
       CMM_ORDER_NO8 = 1,       /* 4s, 2s (no radix 8), odd primes ascending      */
       CMM_ORDER_ODDFIRST = 2,  /* odd primes descending first, then 8s, 4s, 2s  */
       CMM_ORDER_ODDDESC = 3 }; /* 8s, 4s, 2s, then odd primes descending        */
int cmm_grid_create_sched(int n1, int n2, int n3, const double* rvecs, const int* sched, cmm_grid** out);
/* The plan's schedule (sched[5] as above, the plane entry being the forced
 * staging flag) and, optionally, its radices [3][16] (0 past the last stage). */
int cmm_grid_schedule(const cmm_grid* grid, int* sched, int* radices);
/* Smallest `nslot` of the partial-sum arrays d_part / d_ls_part: every pass
 * writes at most this many slots per instance (one per x-plane or column
 * tile); a larger nslot works and only costs the reductions. */
int cmm_part_slots(const cmm_grid* grid);
/* Number of stored frequencies per instance (N1*N2*H3) and H3. */
int cmm_grid_spectrum_size(const cmm_grid* grid, long long* nspec, int* h3);
/* Frequency indices (0..N-1 per axis) at each stored position:
 * k1[N1], k2[N2], k3[H3] (host arrays). */
int cmm_spectrum_index(const cmm_grid* grid, int* k1, int* k2, int* k3);
/* Largest batch-independent shared-memory request of the fused plane pass
 * with `nslot` fields (bytes), for capacity checks. */
int cmm_plane_smem_bytes(const cmm_grid* grid, int nslot, size_t* bytes);

/* Lennard-Jones external potential with Lorentz-Berthelot mixing, per-axis
 * minimum image, R = sqrt(r^2 + 1e-16), cut-and-shifted at `cutoff`, summed
 * over host atoms in file order; then capped: non-finite or > v_cap -> v_cap.
 * Replaces get_external_potential / lennard_jones
 * (cmmdft/extpot_calculator.py:156-222) and the capping in
 * FreeEnergy.add_external_potential (cmmdft/functionals.py:247-251).
 * d_pos: natom x 3 (recentred), d_type: natom type ids, d_type_sig/eps: per type.
 * Output d_V: [N1][N2][N3]. */
int cmm_extpot_lj(const cmm_grid* grid, const double* d_pos, const int* d_type, int natom,
                  const double* d_type_sig, const double* d_type_eps, int ntype,
                  double guest_sig, double guest_eps, double cutoff, double v_cap,
                  double* d_V, void* stream);
/* Form of cmm_extpot_lj for the rest of the process: 0 = by size (default:
 * the cell-list form for orthorhombic cells whose tiles reach under half of
 * the atoms, at least 1024 atoms, and every axis at least three bins of
 * edge cutoff / 2), 1 = the cell-list form wherever the cell allows it,
 * 2 = the all-atom form.  The cell-list form stages, per tile of 4 x 8 x 8
 * grid points, the atoms within the cutoff of the tile in shared memory and
 * sums them in bin order instead of file order (the same pairs; the sum's
 * rounding differs).  Process-wide, not per grid or thread. */
int cmm_extpot_set_mode(int mode);
/* Orientation-averaged external potential of a rigid multi-site guest.
 * Replaces effective_potential_vectorized as generate_effective_potential
 * calls it (cmmdft/extpot_calculator.py:569-655): at every grid point p the
 * guest (guest_pos: nsite x 3 in its own frame, guest_mass: nsite) is moved
 * to p, centred on its centre of mass, turned by each of the nrot matrices
 * d_rot [nrot][3][3] (row-major, applied as R x) and put back; each site's LJ
 * sum over the host atoms uses the site's own sigma/epsilon (guest_sig,
 * guest_eps: nsite, mixed as in cmm_extpot_lj).  Site potentials are
 * rounded to float32 and summed there, scaled by float32(-beta), and the
 * weighted log-sum-exp over rotations (weights d_w [nrot]) is taken in
 * float64 as scipy.special.logsumexp does; d_V = -lse / beta, NaN ->
 * v_limit.  No cap is applied (the caller caps as cmm_extpot_lj does).
 * nsite <= 8, nsite * ntype <= 128.  Up to 6144 rotations the per-point
 * rotation energies stay in shared memory; above that (Lebedev degree >= 27)
 * they go to a stream-ordered global scratch (1 GiB, or 1184 points' rows
 * where that is more), the points taken in chunks that fit it, with the same arithmetic and reduction order.
 * Synchronous. */
int cmm_extpot_rot(const cmm_grid* grid, const double* d_pos, const int* d_type, int natom,
                   const double* d_type_sig, const double* d_type_eps, int ntype,
                   const double* guest_pos, const double* guest_mass, const double* guest_sig,
                   const double* guest_eps, int nsite, const double* d_rot, const double* d_w, int nrot,
                   double cutoff, double beta, double v_limit, double* d_V, void* stream);
/* LJ potential and derivatives of one guest atom type on an n1 x n2 x n3
 * grid over the cell (rvecs row-major, points as Grid.points), the eight
 * channels of get_external_potential_derivatives
 * (cmmdft/extpot_calculator.py:264-338): V, dV/dx, dV/dy, dV/dz, d2V/dxdy,
 * d2V/dxdz, d2V/dydz, d3V/dxdydz, with V and the first derivatives clipped
 * to +-v_max (the reference uses 1e6 kJ/mol), the cross derivatives zeroed
 * where V > v_max, and the derivatives scaled by the axes' `spacings`.
 * d_out: [8][n1][n2][n3].  Synchronous. */
int cmm_extpot_lj_deriv(const double* rvecs, int n1, int n2, int n3, const double* spacings,
                        const double* d_pos, const int* d_type, int natom, const double* d_type_sig,
                        const double* d_type_eps, int ntype, double guest_sig, double guest_eps,
                        double cutoff, double v_max, double* d_out, void* stream);
/* cmm_extpot_rot with each site potential interpolated tricubically
 * (Interpolator.tricubic_interpolation, cmmdft/extpot_calculator.py:391-549)
 * from channel tables d_tab [ntab][8][fine_n0][fine_n1][fine_n2] (as
 * cmm_extpot_lj_deriv writes them); site s reads table site_tab[s]; the cell
 * of a site position q is floor((q - origin) / spacing) with periodic
 * corner indices.  Replaces ExternalPotential.generate_potential with
 * interpolate=True (cmmdft/functionals.py:1032-1055).  Any nrot, as
 * cmm_extpot_rot.  Synchronous. */
int cmm_extpot_rot_interp(const cmm_grid* grid, const double* d_tab, int ntab, const int* fine_n,
                          const double* origin, const double* spacing, const double* guest_pos,
                          const double* guest_mass, const int* site_tab, int nsite, const double* d_rot,
                          const double* d_w, int nrot, double beta, double v_limit, double* d_V, void* stream);

/* Unnormalised 3D real-to-half-complex FFT and its inverse in the plan's
 * spectrum layout (scipy.fft.fftn / ifftn*N as used by Grid.fft/ifft,
 * cmmdft/system.py:310-332, without the reference's phase factor, which
 * cancels in every product the solve forms).  `batch` instances. */
int cmm_rfft3d(const cmm_grid* grid, int batch, const double* d_in, double* d_spec, void* stream);
int cmm_irfft3d(const cmm_grid* grid, int batch, double* d_spec, double* d_out, void* stream);
/* (cmm_irfft3d overwrites d_spec with intermediate data.) */

/* Plane passes alone: y/z real-to-half-complex transform of real fields
 * into yz-spectra, and the inverse (unnormalised). */
int cmm_rfft_yz(const cmm_grid* grid, int batch, const double* d_in, double* d_spec, void* stream);
int cmm_irfft_yz(const cmm_grid* grid, int batch, const double* d_spec, double* d_out, void* stream);

/* Mean-field attraction kernel spectrum: the sampled cut-and-shifted LJ
 * potential U(r) of MFAFunctional.generate_potential_lj
 * (cmmdft/functionals.py:878-910), transformed and folded with the Lanczos
 * factor, the reference's phase exp(i pi scalprod), the cell volume and the
 * FFT normalisations, then Hermitian-symmetrised, so that
 * C1_mfa = irfft3d(rho_hat * K) reproduces MFAFunctional.derive
 * (cmmdft/functionals.py:912-926).  rep = 1 (no tail corrections) or the
 * supercell repetition (2 -> tailcorrections=True, functionals.py:794-796).
 * d_work must hold (rep*N1)(rep*N2)(rep*N3) doubles plus the supercell
 * spectrum; query with d_kst = NULL and work_bytes receiving the size.
 * Output d_kst: double2 [N1][N2][H3] in the x-DIF/y/z position layout used
 * by the column passes.  *vdw_a receives 0.5 * integral U (compute_vdw_a). */
int cmm_mfa_kernel(const cmm_grid* grid, double sigma, double epsilon, double cutoff,
                   double rmin, double limit_potential, int rep, double* d_kst,
                   double* d_work, size_t* work_bytes, double* vdw_a, void* stream);

/* Functional pipeline for `batch` densities given their yz-spectra d_rhohat:
 *   column pass: rho_hat -> analytic FMT weights -> n0, n3, nv2 spectra
 *   plane pass : inverse, White-Bear/FMT dPhi/dn, forward of 5 fields
 *   column pass: back-convolution sum w_a dPhi_a / (beta N) + rho_hat * K_mfa
 * writing d_chat = yz-spectrum of C1 - V (HardSphere.derive + MFA.derive,
 * cmmdft/functionals.py:489-609, 912-926).  d_wtab: weight table from
 * cmm_fmt_weights for this grid and R, or NULL.  want: bit 0 = C1 spectrum,
 * bit 1 = free-energy sums (PHI, MFA), bit 2 = n3 maximum, bit 3 = the
 * weighted densities themselves into d_wd (real fields [nf][batch][N1][N2][N3],
 * nf = 5, +1 with CMM_WDA, +6 with CMM_TENSOR; n0, n3, nv2 x/y/z, WDA, tensor
 * xx, xy, xz, yy, yz, zz), the input of the cmm_ls_* line search.
 * wda: WDA part (with version | CMM_WDA), else NULL; it adds one weighted
 * density and one back-convolution field.  CMM_TENSOR adds the six tensor
 * weighted densities and their back-convolution.
 * d_work: 12 spectra of batch instances (24 with CMM_TENSOR).
 * d_part: [batch][CMM_NSTAT][nslot].
 * With CMM_NOHS (the MFA convolution alone) only want = 1 is accepted: the
 * free-energy sums, the n3 maximum and the weighted densities belong to the
 * hard-sphere passes, so any of want bits 1-3 returns CMM_ERR_ARG. */
int cmm_fmt_c1(const cmm_grid* grid, int batch, const int* d_active, double R, double beta,
               int version, const cmm_wda_eos* wda, const double* d_kst, const double* d_wtab,
               const double* d_rhohat, double* d_chat, double* d_work, double* d_part, int nslot,
               int want, double* d_wd, void* stream);

/* Table of the scalar FMT weights (kw0, kw3 of _init_weight_functions,
 * cmmdft/functionals.py:421-455) in the column-pass layout: double2
 * [N1][N2][H3].  Passing it as d_wtab to cmm_fmt_c1 replaces the per-element
 * evaluation of sin/cos (same formulas, evaluated once per grid and radius). */
int cmm_fmt_weights(const cmm_grid* grid, double R, double* d_wtab, void* stream);

/* Fused plane pass of one static Picard step (Picard.update_rho_static,
 * cmmdft/solver.py:392-401, with get_new_rho :128-129):
 *   C1 = irfft(chat) + V; G = beta exp(-beta C1) f;  RES2 += (G - rho)^2
 *   rho' = (1-a) rho + a G; rho' < thr -> 0;  writes rho', its spectrum and
 *   the reductions N, IUE, NONFIN, FID, FEXT of rho'.
 * d_params: [batch][4] = {fugacity f, a, mu, unused}.  d_V stride vstride.
 * Also the DER sum of the input density (Solver._check_convergence,
 * solver.py:200-205) with the Solver tolerances a_tol, r_tol (solver.py:25-26,
 * defaults 1e-6 and 1e-4; both must be >= 0). */
int cmm_picard_static_step(const cmm_grid* grid, int batch, const int* d_active,
                           const double* d_params, double beta, double lambda3, double thr,
                           double a_tol, double r_tol, const double* d_chat, const double* d_rho, const double* d_V,
                           long long vstride, double* d_rho_out, double* d_rhohat_out,
                           double* d_part, int nslot, void* stream);

/* Residual plane pass (Anderson.update_rho / _save_previous_rhos,
 * cmmdft/solver.py:527-579): C1 = irfft(chat) + V; G = beta exp(-beta C1) f;
 * writes r = G - rho to d_r_out; reductions RES2, GNONFIN, DER and the Gram row
 * sum r * r_j over `nhist` stored residuals d_hist[j] (HOST array of
 * device pointers, instance stride hstride); a_tol, r_tol as in
 * cmm_picard_static_step. */
int cmm_residual_step(const cmm_grid* grid, int batch, const int* d_active,
                      const double* d_params, double beta, double lambda3, double a_tol,
                      double r_tol, const double* d_chat,
                      const double* d_rho, const double* d_V, long long vstride,
                      double* d_r_out, const double* const* d_hist, int nhist,
                      long long hstride, double* d_part, int nslot, void* stream);

/* Mix plane pass: rho' = sum_j c[b][j] field_j (up to 12 fields), clipped
 * (CMM_CLIP_*), written with its spectrum and the reductions N, IUE (against
 * d_ref), NONFIN, FID, FEXT.  Covers the Picard hybrid trial densities and
 * mixing (solver.py:403-457) and the Anderson mixing (solver.py:593-598).
 * thr is the CMM_CLIP_PICARD threshold.  d_coef: [batch][12] (device);
 * d_fields / fstride: HOST arrays of nfield device pointers / instance strides. */
int cmm_mix_step(const cmm_grid* grid, int batch, const int* d_active, const double* d_coef,
                 const double* const* d_fields, const long long* fstride, int nfield,
                 int clip, double thr, double lambda3, const double* d_ref, long long refstride,
                 const double* d_V, long long vstride, double* d_rho_out,
                 double* d_rhohat_out, double* d_part, int nslot, void* stream);

/* Reduce d_part [batch][CMM_NSTAT][nslot] over slots into d_stats
 * [batch][CMM_NSTAT] for the stats whose bit is set in `mask` (max for
 * CMM_STAT_N3MAX, sums otherwise). */
int cmm_stats_finalize(int batch, const int* d_active, const double* d_part, int nslot,
                       unsigned mask, double* d_stats, void* stream);

/* Hybrid Picard line search (Picard.update_rho_hybrid and _get_alpha_max,
 * cmmdft/solver.py:150-165, 403-433) without transforms of the trial
 * densities: weighted densities are linear in the density, so Omega(rho +
 * alpha r) follows from the weighted densities of rho (cmm_fmt_c1, want bit
 * 3) and of r pointwise; the MFA energy is quadratic and N, F_ext linear in
 * alpha.  d_ls_part: [batch][CMM_NLS][nslot] partial sums, initialised once
 * by the caller (0, and -inf in the CMM_LS_N3MAX_G slots); every call
 * rewrites the same slots.
 *
 * cmm_ls_prepare: the weighted densities of the residuals d_r (real fields)
 * into d_wd_r, the MFA sums of r against the yz-spectra d_rhohat of rho, and
 * max (n3(rho) + n3(r)) with the n3 field of d_wd_rho.  d_rhat: scratch of
 * one yz-spectrum per instance; d_work as cmm_fmt_c1. */
int cmm_ls_prepare(const cmm_grid* grid, int batch, const int* d_active, double R, int version,
                   const cmm_wda_eos* wda, const double* d_kst, const double* d_wtab, const double* d_r,
                   const double* d_rhohat, const double* d_wd_rho, double* d_rhat, double* d_work,
                   double* d_wd_r, double* d_ls_part, int nslot, void* stream);
/* cmm_ls_omega: alpha_max = min(|(1 - a) / ((g - a) + 1e-16)|, 1) per
 * instance (a = d_n3a[b * n3a_stride], the max n3 of rho; g =
 * CMM_LS_N3MAX_G), written to d_alpha[b]; then the pointwise sums of
 * CMM_LS_SUM_R .. WDA at alpha_i = coef[i] * alpha_max, i < 3. */
int cmm_ls_omega(const cmm_grid* grid, int batch, const int* d_active, const double* d_n3a,
                 long long n3a_stride, double c0, double c1, double c2, double R, double lambda3, int version,
                 const cmm_wda_eos* wda, const double* d_rho, const double* d_r, const double* d_V,
                 long long vstride, const double* d_wd_rho, const double* d_wd_r, double* d_ls_part,
                 int nslot, double* d_alpha, void* stream);
/* Reduce d_ls_part over slots into d_ls [batch][CMM_NLS] (max for
 * CMM_LS_N3MAX_G, sums otherwise). */
int cmm_ls_finalize(int batch, const int* d_active, const double* d_ls_part, int nslot, double* d_ls,
                    void* stream);

/* ---------------------------------------------------------------------
 * Native batched solve: the control flow of Solver._solve with the
 * Picard static and hybrid and the (hybrid-)Anderson updates
 * (cmmdft/solver.py:236-345, 392-457, 515-604) for `batch` chemical
 * potentials on one functional, run
 * in C++ around the kernels above (one read-back per decision point).
 * Equivalent to the Python driver cmmdft_b200.batch.BatchSolve, which
 * remains its specification.
 * ------------------------------------------------------------------- */
typedef struct cmm_functional_desc {
  const cmm_grid* grid;
  double R, beta, lambda3;
  int version;                  /* CMM_FMT / MFMT / WBII | ANTISYM | TENSOR | WDA */
  const cmm_wda_eos* wda;       /* with CMM_WDA, else NULL */
  const double* d_kst;          /* MFA kernel spectrum */
  const double* d_wtab;         /* weight table or NULL */
  const double* d_V;            /* external potential [N1][N2][N3] */
} cmm_functional_desc;

enum { CMM_SOLVE_HYBRID = 1, CMM_SOLVE_ANDERSON = 2, CMM_SOLVE_HYBRIDANDERSON = 3,
       CMM_SOLVE_STATIC = 4 /* Picard.update_rho_static, solver.py:392-401 */ };
enum { CMM_CRIT_RES = 0, CMM_CRIT_RIUE = 1, CMM_CRIT_DER = 2 };
/* Anderson coefficients: the reference's SLSQP (solver.py:585-591, restated
 * in cmm_anderson_slsqp) or the exact minimiser of ||sum a_i r_i|| on the
 * simplex (fewer steps; trajectories then differ from the reference's). */
enum { CMM_COEF_SLSQP = 0, CMM_COEF_EXACT = 1 };

typedef struct cmm_solve_opts {
  int method;                   /* CMM_SOLVE_* */
  int nsteps, m;                /* step limit, Anderson history depth */
  int ncrit, crit[3];           /* criteria, all must hold */
  double thr[3];
  double alpha_mix, damping, delta, damping_max, damping_min, damping_up, damping_down;
  int adaptive_damping;
  int divergence_guard;         /* retire instances whose RES rises past 1e6 x best */
  double a_tol, r_tol;          /* DER tolerances */
  double ls_thresh;             /* 1 kJ/mol: line-search fallback threshold (Hartree) */
  double kjmol;                 /* 1 kJ/mol in Hartree */
  int coefs;                    /* CMM_COEF_* */
  double picard_thr;            /* static Picard: densities below this become 0 (1e-10 angstrom^-3 in the
                                   caller's length unit, solver.py:398) */
  int device_loop;              /* static Picard: 1 = the per-instance decisions in a device kernel and the
                                   step replayed as a CUDA graph (the host reads one counter every 4 steps),
                                   0 = decisions on the host after every step; same results */
} cmm_solve_opts;

/* Buffers of one solve (device, except the h_* pinned host arrays).
 * npts = N1*N2*N3, S = 2*N1*N2*H3 doubles (one yz-spectrum), nwd as
 * cmm_fmt_c1's want bit 3, nwork = 12 (24 with CMM_TENSOR). */
typedef struct cmm_solve_ws {
  double* ring;                 /* [m][B][npts] densities */
  double* rres;                 /* [m][B][npts] residuals */
  double* trial;                /* [B][npts] */
  double* rho0;                 /* [B][npts] initial densities (input) */
  double* result;               /* [B][npts] final densities (output) */
  double* spec_ring;            /* [m][B][S] */
  double* wd_ring;              /* [m][nwd][B][npts] */
  double* wd_r;                 /* [nwd][B][npts] */
  double* rhat, *chat, *chat2, *that;   /* [B][S] each */
  double* work;                 /* [nwork][B][S] */
  double* part;                 /* [B][CMM_NSTAT][nslot], N3MAX slots -inf */
  double* stats;                /* [B][CMM_NSTAT] */
  double* params;               /* [B][4] */
  double* coef;                 /* [B][12] */
  int* active;                  /* [B] */
  double* ls_part;              /* [B][CMM_NLS][nslot], 0 and -inf in CMM_LS_N3MAX_G */
  double* ls;                   /* [B][CMM_NLS] */
  double* ls_alpha;             /* [B] */
  int nslot;
  double* h_stats;              /* pinned [B][CMM_NSTAT] */
  double* h_ls;                 /* pinned [B][CMM_NLS] */
  double* h_alpha;              /* pinned [B] */
  void* h_stage;                /* pinned staging of uploads, cmm_solve_stage_bytes(B) */
  double* h_result;             /* optional pinned [B][npts]: each final density is copied here on a
                                   side stream as soon as its instance finishes (NULL: none) */
} cmm_solve_ws;

typedef struct cmm_solve_out {
  double* N;                    /* [B] loading (integral of rho) */
  double* omega;                /* [B] grand potential of the last density */
  int* converged, *steps, *diverged, *failed;   /* [B]; failed: non-finite on every retry */
  double* history;              /* optional [B][nsteps + 2][CMM_HISTORY_COLS] per step: N, RES, RIUE, the
                                   grand potential of the step's last evaluation, and sqrt(DER sum / npts)
                                   (solver.py:208-222); or NULL */
  long long launches;           /* kernel launches issued */
  long long omega_evals;
  double* pipe_log;             /* optional [pipe_cap][3]: (want, active instances, ms) per full
                                   functional-pipeline launch, CUDA-event timed (NULL: not timed) */
  int pipe_cap, pipe_n;
  double* cf;                   /* optional [B]: final correction factor of each instance (1, halved per
                                   non-finite restart, solver.py:335-345), or NULL */
} cmm_solve_out;
#define CMM_HISTORY_COLS 5

/* ---------------------------------------------------------------------
 * Derivatives at a converged density (implicit adjoint; the reference has no
 * derivatives -- its users difference whole solves).
 * ------------------------------------------------------------------- */
/* Spectrum of A v, A = d C1 / d rho the Hessian of the excess free energy
 * (hard-sphere + MFA, + the WDA part with CMM_WDA; C1 in Hartree, so A v is
 * in Hartree per density unit), for `batch` yz-spectra d_vhat.  d_wd_rho:
 * the real-space weighted densities of rho [nwd][B][npts] stored by
 * cmm_fmt_c1 with want bit 3; the hard-sphere and EOS second derivatives
 * are taken there.  wda: the WDA part's EOS with CMM_WDA, else NULL.
 * transpose = 1: A^T v, with the caller passing the conjugate MFA spectrum
 * as d_kst (A is not symmetric: the reference's MFA kernel is translated by
 * its spectrum phase, and where n3 is clipped dPhi/dn3 still varies with
 * the other densities; the WDA part is symmetric).  d_work: nwork spectra
 * as for cmm_fmt_c1. */
int cmm_fmt_hvp(const cmm_grid* grid, int batch, const int* d_active, double R, double beta, int version,
                const cmm_wda_eos* wda, int transpose, const double* d_kst, const double* d_wtab,
                const double* d_wd_rho, const double* d_vhat, double* d_out_hat, double* d_work, void* stream);

/* Parameter derivatives of the capped LJ external potential (arguments as
 * cmm_extpot_lj): d_dV [2 + 2 ntype][npts], rows dV/d(guest eps),
 * dV/d(guest sigma), dV/d(eps_t) for each host type, dV/d(sigma_t) for each
 * host type; zero where the potential is capped.  ntype <= 8. */
int cmm_extpot_lj_grad(const cmm_grid* grid, const double* d_pos, const int* d_type, int natom,
                       const double* d_type_sig, const double* d_type_eps, int ntype, double guest_sig,
                       double guest_eps, double cutoff, double v_cap, double* d_dV, void* stream);

/* d_part[(w K + k) nchunk + c] = partial sums over chunk c of the n points of
 * W[w] * D[k] (row strides ldw, ldd); the caller sums over c. */
int cmm_contract(const double* d_W, long long ldw, int nw, const double* d_D, long long ldd, int K, long long n,
                 double* d_part, int nchunk, void* stream);

/* Vector steps of the batched BiCGSTAB on (I + c S A^T S) y = rhs,
 * S = diag(sqrt(max(rho, 0))), fields [batch][npts], scalars d_sc
 * [batch][CMM_BICG_NS] (CMM_BICG_FIRST = 1 before the first step):
 *   op 0: out = S x
 *   op 1: out = x + c S y, partial dots (out . a, out . out)
 *   op 2: out (p) = x (r) + beta (out - omega y (v))
 *   op 3: out (s) = x (r) - alpha y (v)
 *   op 4: out (solution) += alpha x (p) + omega y (s); out2 (r) = y - omega a (t);
 *         partial dots (rhat . r, r . r)
 * Partial dots go to d_part [batch][2][nblk]. */
enum { CMM_BICG_RHO = 0, CMM_BICG_ALPHA = 1, CMM_BICG_OMEGA = 2, CMM_BICG_BETA = 3, CMM_BICG_D0 = 4,
       CMM_BICG_D1 = 5, CMM_BICG_RR = 6, CMM_BICG_FIRST = 7, CMM_BICG_NS = 8 };
int cmm_bicg_vec(int op, long long npts, int batch, const int* d_active, const double* d_rho, const double* d_sc,
                 double c, const double* d_x, const double* d_y, const double* d_a, double* d_out, double* d_out2,
                 const double* d_rhat, double* d_part, int nblk, void* stream);
/* Sum the partial dots (fixed order) and advance the scalars: stage 0 after
 * op 4 (rho, beta, r . r), 1 after the product of p (alpha), 2 after the
 * product of s (omega). */
int cmm_bicg_scalars(int batch, const int* d_active, const double* d_part, int nblk, double* d_sc, int stage,
                     void* stream);

/* Anderson mixing coefficients of one instance as Anderson.update_rho_Anderson
 * computes them (cmmdft/solver.py:581-591): scipy's SLSQP from a = 1/n with
 * tol 1e-10 on sum_res(a) = ||sum_i a_i r_i||, bounds [0, 1], sum a = 1 --
 * restated on the host from Kraft's algorithm with scipy's 2-point finite
 * differences, the objective taken as sqrt(a^T G a) from the Gram matrix
 * gram [n][n] = <r_i, r_j> (oldest residual first, n <= 8).  *mode receives
 * SLSQP's exit mode (0 converged, 8 no descent direction, 9 iteration limit);
 * alpha is SLSQP's last iterate in every case, as the reference uses it. */
int cmm_anderson_slsqp(const double* gram, int n, double* alpha, int* mode, int* nit);

/* The line search's SLSQP fallback (solver.py:437-447) is delegated to the
 * caller: minimise Omega((1-a) rho + a G) over a in [0.01, 0.9] alpha_max for
 * instance b, rho in ring slot s_prev; returns 0 and alpha (and the last
 * Omega evaluated) on success. */
typedef int (*cmm_fallback_fn)(void* ctx, int b, int s_prev, double alpha_max, double* alpha, double* omega);

size_t cmm_solve_stage_bytes(int batch);
int cmm_solve_batched(const cmm_functional_desc* fn, const cmm_solve_opts* opt, int batch, const double* mu,
                      const double* fug, const double* cf0, const cmm_solve_ws* ws, cmm_solve_out* out,
                      cmm_fallback_fn fallback, void* fallback_ctx, void* stream);

/* Allocation-free variant of cmm_fmt_c1 (no counterpart in the reference,
 * which allocates freely in numpy).  For callers that cannot allocate device
 * memory where they evaluate the functional -- plugin hosts that forbid
 * allocation inside a solve callback, integrations under a fixed device
 * memory budget, bindings whose runtime cannot own a CUDA allocation.
 * The scratch (twelve intermediate spectra and the partial sums) lives in one
 * static device array of CMM_NOALLOC_SCRATCH_BYTES that every GPU loading
 * the library holds until exit; batches larger than
 * cmm_fmt_c1_noalloc_capacity(grid) are rejected with CMM_ERR_WORKSPACE.
 * The first call on a device looks up the array's address (make it before
 * any stream capture); the address is kept per device index for the life of
 * the process, so a cudaDeviceReset (or anything else that destroys and
 * re-creates the device's primary context) invalidates it, and this entry
 * point must not be called on that device afterwards.  All calls share the
 * array and it keeps the last call's contents: calls that overlap on the GPU
 * race.  Outputs as cmm_fmt_c1; d_stats [batch][CMM_NSTAT] receives the PHI /
 * MFA / N3MAX sums requested by `want` (may be NULL when want == 1), and
 * CMM_NOHS accepts want = 1 only, as in cmm_fmt_c1.  The tensor versions
 * (CMM_TENSOR) need twice the scratch and return CMM_ERR_UNSUPPORTED. */
#define CMM_NOALLOC_SCRATCH_BYTES (32u << 20)
size_t cmm_fmt_c1_noalloc_capacity(const cmm_grid* grid);
int cmm_fmt_c1_noalloc(const cmm_grid* grid, int batch, const int* d_active, double R, double beta,
                       int version, const cmm_wda_eos* wda, const double* d_kst, const double* d_wtab,
                       const double* d_rhohat, double* d_chat, double* d_stats, int want, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* CMMDFT_B200_H */
