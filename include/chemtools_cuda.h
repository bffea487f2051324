/* chemtools_cuda.h -- C ABI of the B200-native grid-evaluation library.
 *
 * Drop-in boundary for ChemToolsCUDA's grid-evaluation hot path.  Every entry
 * point is extern "C", takes plain pointers and sizes, and returns 0 on
 * success or a negative CTC_ERR_* code; ctc_last_error() then describes the
 * failure (per calling thread).  Nothing here allocates device memory that
 * outlives the molecule handle: each handle owns its device copy of the basis
 * and density matrix and its scratch.  The library keeps, per process, only
 * which kernels have been configured on which device (their shared-memory
 * limits, set once per device) and the no-allocation entry point's fixed
 * array (ctc_eval_local_noalloc).
 *
 * Device-pointer entry points are stream-ordered on the stream passed in
 * (NULL = legacy default stream) and return before the work finishes; they
 * do not synchronise.  A failure that a kernel detects on the device (a
 * bounded wait of the tensor-core pipeline running out) is recorded in the
 * molecule's status word and reported as CTC_ERR_DEVICE by the next call on
 * that molecule whose copy of the word has landed, or at once by
 * ctc_molecule_sync_status.  Use one stream at a time per molecule.  The
 * *_host variants take host pointers, copy inputs and outputs themselves and
 * return after the results are in host memory (and report device failures
 * of their own kernels).
 *
 * Layouts: points are row-major (N, 3) doubles; gradients (N, 3); Hessians
 * (N, 3, 3); scalar descriptors (N,).  AO functions follow the reference's
 * order: shells in input order, segments in order, and within a segment the
 * Cartesian order xx,yy,zz,xy,xz,yz (d), xxx,yyy,zzz,xyy,xxy,xxz,xzz,yzz,yyz,xyz
 * (f), zzzz,yzzz,...,xxxx (g), or the pure order c0,c1,s1,c2,s2,... .
 */
#ifndef CHEMTOOLS_CUDA_B200_H_
#define CHEMTOOLS_CUDA_B200_H_

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- error codes --------------------------------------------------------------------------- */
#define CTC_OK 0
#define CTC_ERR_INVALID (-1)     /* bad argument (null pointer, size, angular momentum, ...) */
#define CTC_ERR_CUDA (-2)        /* a CUDA runtime call failed */
#define CTC_ERR_UNSUPPORTED (-3) /* feature not available for this input / device */
#define CTC_ERR_NOMEM (-4)       /* device or pinned-host allocation failed */
#define CTC_ERR_DEVICE (-5)      /* a kernel reported an error through its status word */

/* ---- precision of the Phi*D contraction ------------------------------------------------------ */
#define CTC_PREC_FP64 0      /* FP64 throughout (double-precision matrix units) */
#define CTC_PREC_TC_SPLIT 1  /* INT8 tensor cores, operands split into int8 digits (5 for the AO rows, 5 for D), exact int32 accumulation */

typedef struct ctc_molecule ctc_molecule; /* opaque handle */

/* Contracted Gaussian basis in the reference's generalised-contraction form
 * (include/contracted_shell.h:39-44): shell s has nprim[s] exponents shared by
 * nseg[s] segments; segment g has angular momentum angmoms[...] in the fchk
 * code (0 s, 1 p, 2 Cartesian d, -2 pure d, 3/-3 f, 4/-4 g) and coefficients
 * coeffs[off + g*nprim[s] + k] of L2-normalised primitives.  shell_atom may be
 * NULL, in which case shells are attached to the atom at their centre. */
typedef struct {
  int32_t nshell;
  const double* centers;     /* [nshell][3] bohr */
  const int32_t* shell_atom; /* [nshell] or NULL */
  const int32_t* nprim;      /* [nshell] */
  const int32_t* nseg;       /* [nshell] */
  const int32_t* angmoms;    /* [sum nseg] */
  const double* exps;        /* [sum nprim] */
  const double* coeffs;      /* [sum nseg*nprim] */
} ctc_basis;

/* Output slots of the local-descriptor evaluation.  A NULL slot is not
 * computed; the kernels then skip the derivatives and products that only it
 * needs. */
typedef struct {
  double* rho;          /* (N)     electron density */
  double* grad;         /* (N,3)   gradient of rho */
  double* hess;         /* (N,3,3) Hessian of rho */
  double* lap;          /* (N)     Laplacian of rho */
  double* tau_pd;       /* (N)     positive-definite kinetic-energy density */
  double* tau_alpha;    /* (N)     tau_pd + alpha * lap */
  double* rdg;          /* (N)     reduced density gradient */
  double* shannon;      /* (N)     rho * ln(rho) */
  double* weizsacker;   /* (N)     |grad rho|^2 / (8 rho) */
  double* thomas_fermi; /* (N)     3/10 (3 pi^2)^(2/3) rho^(5/3) */
  double* gge;          /* (N)     thomas_fermi + gge_a * weizsacker + gge_b * lap */
  double* general_ked;  /* (N)     tau_pd + (ked_a - 1)/4 * lap */
} ctc_outputs;

typedef struct {
  double alpha;        /* tau_alpha parameter */
  double gge_a, gge_b; /* general gradient-expansion parameters */
  double ked_a;        /* general(ish) KED parameter */
} ctc_params;

/* ---- molecule ------------------------------------------------------------------------------ */

/* Build a molecule on the current device: basis tables, density matrix D
 * (nbasis x nbasis, row-major, symmetric, host memory), atoms (host).
 * Replaces the IOData/MolecularBasis set-up of the reference
 * (include/iodata.h:34-38, src/iodata.cpp:15-211) and the constant-memory
 * upload (src/basis_to_gpu.cu:16-166, include/basis_to_gpu.cuh:42). */
int ctc_molecule_create(const ctc_basis* basis, int32_t natom, const double* atom_xyz,
                        const double* atom_charges, const double* D, int32_t nbasis,
                        ctc_molecule** out);
int ctc_molecule_destroy(ctc_molecule* mol);
int ctc_molecule_nbasis(const ctc_molecule* mol);
int ctc_molecule_natom(const ctc_molecule* mol);

/* Replace D from device memory (nbasis x nbasis, row-major, symmetric):
 * stream-ordered, a permuting copy on the device with no host round trip.
 * Replaces the per-call cublasSetMatrix uploads (e.g.
 * src/evaluate_density.cu:777). */
int ctc_molecule_set_density_matrix(ctc_molecule* mol, const double* d_D, void* stream);

/* Move the atoms (host (natom,3)); the shells move with their atoms. */
int ctc_molecule_set_coordinates(ctc_molecule* mol, const double* atom_xyz);

/* Make every table the evaluation needs resident on the device now (the
 * split-precision copy of D included).  Idempotent.  Replaces
 * Molecule::basis_set_to_constant_memory (src/pymolecule.cu:25-32). */
int ctc_molecule_prepare(ctc_molecule* mol, int32_t precision);

/* ---- Gaussian formatted checkpoint files ----------------------------------
 * Replaces chemtools::get_molecular_basis_from_fchk (src/iodata.cpp:15-211),
 * which reads the file through the Python iodata package, and the Molecule(str)
 * constructor built on it (src/pymolecule.cu:18-23).  The density matrix is the
 * MO one-particle density matrix (C occ) C^T as the reference forms it
 * (src/iodata.cpp:157-160); basis functions keep Gaussian's order within each
 * shell, which is the order of the reference's kernels. */
typedef struct ctc_fchk ctc_fchk;

typedef struct {
  ctc_basis basis;              /* arrays owned by the ctc_fchk */
  int32_t natom;
  const double* atom_xyz;       /* [natom][3], bohr */
  const double* atom_charges;   /* [natom] nuclear charges */
  const int32_t* atomic_numbers;/* [natom] */
  int32_t nbasis;
  int32_t nalpha, nbeta;        /* electrons */
  const double* density;        /* [nbasis][nbasis] */
} ctc_fchk_view;

int ctc_fchk_load(const char* path, ctc_fchk** out);
int ctc_fchk_view_get(const ctc_fchk* f, ctc_fchk_view* out);
void ctc_fchk_destroy(ctc_fchk* f);
/* ctc_molecule_create with the contents of an .fchk file. */
int ctc_molecule_create_from_fchk(const char* path, ctc_molecule** out);

/* ---- Molden files -----------------------------------------------------------
 * The other wavefunction format the reference's Molecule(str) accepts through
 * iodata (src/pymolecule.cu:18-23, src/iodata.cpp:15-211).  Fills the same
 * ctc_fchk handle as ctc_fchk_load (read it with ctc_fchk_view_get, release it
 * with ctc_fchk_destroy): atoms, [GTO] shells with the [5D]/[5D10F]/[7F]/
 * [5D7F]/[9G] spherical flags, basis functions in the library's order
 * (Molden's Cartesian g order is permuted), and the density matrix
 * sum_i occ_i c_i c_i^T over the [MO] orbitals with their occupations. */
int ctc_molden_load(const char* path, ctc_fchk** out);

/* ---- AIM wavefunction files (.wfn, .wfx) ---------------------------------------
 * The primitive-based formats the reference's Molecule(str) also accepts
 * through iodata (src/pymolecule.cu:18-23).  Every distinct (centre, l,
 * exponent) of the file's primitives becomes a one-primitive Cartesian shell;
 * orbital coefficients, which multiply unnormalised primitives in these
 * files, are rescaled to the library's normalised functions, and the density
 * matrix is sum_i occ_i c_i c_i^T.  The .wfx form is recognised by its tags.
 * Primitive types 1-20 (s to f); g primitives are refused.  Fills the same
 * ctc_fchk handle as ctc_fchk_load. */
int ctc_wfn_load(const char* path, ctc_fchk** out);

/* ctc_molecule_create from a wavefunction file, by extension: .molden,
 * .molden.input and .mold are read as Molden files, .wfn and .wfx as AIM
 * wavefunction files, anything else as fchk.  Replaces Molecule(str)
 * (src/pymolecule.cu:18-23). */
int ctc_molecule_create_from_file(const char* path, ctc_molecule** out);

/* ---- local descriptors --------------------------------------------------------------------- */

/* All requested local descriptors at N points in one fused pass.  Replaces
 * evaluate_electron_density_on_any_grid (include/evaluate_density.cuh:113),
 * evaluate_electron_density_gradient (include/evaluate_gradient.cuh:95),
 * evaluate_electron_density_hessian (include/evaluate_hessian.cuh:88),
 * evaluate_laplacian (include/evaluate_laplacian.cuh:97),
 * evaluate_positive_definite_kinetic_density and
 * evaluate_general_kinetic_energy_density (include/evaluate_kinetic_dens.cuh:27,45),
 * and compute_reduced_density_gradient, compute_weizsacker_ked,
 * compute_thomas_fermi_energy_density, compute_ked_gradient_expansion_general,
 * compute_general_ked, compute_shannon_information_density
 * (include/evaluate_densbased.cuh:31-103). */
int ctc_eval_local(ctc_molecule* mol, const double* d_points, int64_t npoints, int32_t precision,
                   const ctc_params* params, const ctc_outputs* d_out, void* stream);

/* ctc_eval_local in the FP64 form for callers that cannot allocate device
 * memory during a call (a caller whose own arena holds the device's memory,
 * a run that allocates only at start-up, a process under a fixed
 * device-memory quota).  Has no counterpart in the reference.  It allocates
 * nothing: its scratch is one 64 MiB array compiled into the library, held on
 * every GPU that loads it until the process exits.  At most 1,048,576 points
 * per call, and a basis whose AO block for one 32-point tile does not fit
 * the array is refused; both return CTC_ERR_INVALID with the limit in
 * ctc_last_error().  The first call on a device looks up the array's device
 * address (make it before any stream capture).  All calls share the array:
 * calls that overlap on the GPU race, so serialise them on one stream. */
int ctc_eval_local_noalloc(ctc_molecule* mol, const double* d_points, int64_t npoints,
                           const ctc_params* params, const ctc_outputs* d_out, void* stream);

/* Same with host points and host outputs; copies are inside the call. */
int ctc_eval_local_host(ctc_molecule* mol, const double* h_points, int64_t npoints,
                        int32_t precision, const ctc_params* params, const ctc_outputs* h_out);

/* Descriptors on a cubic grid generated on the device: point (i,j,k) =
 * origin + i*axes[0..2] + j*axes[3..5] + k*axes[6..8], k fastest, outputs in
 * (shape[0], shape[1], shape[2]) C order.  Replaces
 * evaluate_electron_density_on_cubic (include/evaluate_density.cuh:100). */
int ctc_eval_cubic(ctc_molecule* mol, const double* origin, const double* axes,
                   const int32_t* shape, int32_t precision, const ctc_params* params,
                   const ctc_outputs* d_out, void* stream);

/* AO values and derivatives, out (nq, N, nbasis) with nq = 1, 4 or 10 for
 * deriv = 0, 1, 2 (value, x, y, z, xx, xy, xz, yy, yz, zz).  Replaces
 * evaluate_contraction_derivatives (include/evaluate_gradient.cuh:61) and
 * evaluate_contraction_second_derivative (include/evaluate_hessian.cuh:56). */
int ctc_eval_ao(ctc_molecule* mol, const double* d_points, int64_t npoints, int32_t deriv,
                double* d_out, void* stream);

/* ---- electrostatic potential ------------------------------------------------------------- */

/* V(r) = sum_A Z_A/|r - R_A| - sum_{mu nu} D_{mu nu} (mu|1/|r - r'||nu) at N
 * points.  Replaces compute_electrostatic_potential_over_points
 * (include/evaluate_electrostatic.cuh:37).  Shells up to g are supported. */
int ctc_eval_esp(ctc_molecule* mol, const double* d_points, int64_t npoints, double* d_out,
                 void* stream);
int ctc_eval_esp_host(ctc_molecule* mol, const double* h_points, int64_t npoints, double* h_out);

/* Work of the ESP evaluation (no counterpart in the reference; builds the
 * molecule's pair tables if needed): info[0] primitive pairs kept after the
 * point-independent screening, [1] algorithmic FP64 operations per point,
 * sum over those pairs of 2 n_tuv(L) + 2 n_R(L) + 10 (L + 1) with
 * n_tuv(L) = (L+1)(L+2)(L+3)/6 and n_R(L) = sum_{j<=L} n_tuv(j), [2] Hermite
 * coefficients stored, [3] mean L = l_a + l_b of the kept pairs. */
int ctc_molecule_esp_info(ctc_molecule* mol, double* info /* [4] */);

/* ---- adjoint (no counterpart in the reference) --------------------------------------------- */

/* Given v_rho = dL/drho (N) and v_grad = dL/d(grad rho) (N,3, may be NULL)
 * at N points, accumulate (+=) dL/dD (nbasis x nbasis, entries treated as
 * independent) and dL/dR (natom x 3, points and weights held fixed).  Either
 * output may be NULL.  Device pointers, stream-ordered. */
int ctc_adjoint(ctc_molecule* mol, const double* d_points, int64_t npoints, const double* d_v_rho,
                const double* d_v_grad, double* d_dLdD, double* d_dLdR, void* stream);

/* ---- diagnostics ---------------------------------------------------------------------------- */

/* Work counters of the local-descriptor pipeline accumulated since the last
 * reset (no counterpart in the reference): stats[0] tiles, [1] points in
 * tiles, [2] sum of compact AO counts, [3] sum over tiles of rows * kt^2
 * (multiply-adds of the contraction on the screened AO set), [4] kernel
 * launches issued, [5] chunks, [6] milliseconds spent in the contraction
 * kernels and [7] in the AO kernels (both 0 unless profiling is on).
 * Synchronises the device. */
int ctc_molecule_get_stats(ctc_molecule* mol, double* stats /* [8] */);
int ctc_molecule_reset_stats(ctc_molecule* mol);
/* Time the contraction and AO kernels with CUDA events on their stream. */
int ctc_molecule_set_profiling(ctc_molecule* mol, int32_t on);

/* Wait for the stream, then report a failure any kernel of an earlier call on
 * this molecule recorded on the device: CTC_ERR_DEVICE with the cause in
 * ctc_last_error(), or CTC_OK.  Reporting clears the record, and the molecule
 * stays usable.  The reference has no such path: its drivers turn a
 * cudaError_t into a C++ exception (include/cuda_utils.cuh:55-60). */
int ctc_molecule_sync_status(ctc_molecule* mol, void* stream);

/* Limit, in SM clock cycles, of every wait in the tensor-core pipeline
 * (0 = the default of 4e9 cycles, about 2 s).  A kernel whose wait runs out
 * stops issuing work, waits for its own copies in flight, frees its tensor
 * memory, records CTC_ERR_DEVICE in the status word and returns; the
 * molecule stays usable.  A short limit makes the waits run out on purpose
 * (tests of that path); no counterpart in the reference. */
int ctc_molecule_set_wait_limit(ctc_molecule* mol, int64_t cycles);

/* ---- misc ---------------------------------------------------------------------------------- */
const char* ctc_last_error(void);
const char* ctc_version(void);

#ifdef __cplusplus
}
#endif
#endif /* CHEMTOOLS_CUDA_B200_H_ */
