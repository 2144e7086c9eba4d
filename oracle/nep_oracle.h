/*
 * nep_oracle.h -- TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C, double-precision restatement of DMG-MD's NEP force evaluation
 * (NEP4 / NEP5 / NEP-ZBL energy, force and per-atom virial for a periodic
 * box).  It is the checker the tests, the smoke run and the CPU-baseline leg
 * of bench.py compare the CUDA engine against.  Nothing in the product
 * (dmg-md_b200/) links, loads or calls it.
 *
 * Reference anchors (paths inside the DMG-MD project):
 *   potential file parser      src/gpumd_compat/nep.cu:135-415
 *   descriptor + ANN           src/gpumd_compat/nep.cu:569-748,
 *                              src/gpumd_compat/nep_utilities.cuh:169-315
 *   radial force               src/gpumd_compat/nep.cu:756-881
 *   angular partial force      src/gpumd_compat/nep.cu:890-991,
 *                              src/gpumd_compat/nep_utilities.cuh:1296-1491
 *   many-body gather           src/gpumd_compat/potential.cu:81-210
 *   ZBL                        src/gpumd_compat/nep.cu:996-1111,
 *                              src/gpumd_compat/nep_utilities.cuh:378-475
 *   small-box image expansion  src/gpumd_compat/nep.cu:2002-2064,
 *                              src/gpumd_compat/nep_small_box.cuh:96-176
 *   typewise neighbour filter  src/gpumd_compat/nep.cu:503-561
 *
 * Parity is pinned by tests/test_oracle_golden.py (GPUMD 5.9.1 golden
 * vectors of the reference's tests/baseline suite) and by
 * tests/test_oracle_ref_cpu.py (the reference's own FP64 CPU evaluator,
 * NEP3_CPU, compiled from its sources into oracle/_ref/).
 */
#ifndef NEP_ORACLE_H
#define NEP_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct nepo_model nepo_model;

/* Parse a GPUMD-format nep.txt.  Returns NULL and fills err on failure. */
nepo_model* nepo_load(const char* path, char* err, int errlen);
void nepo_free(nepo_model* m);

/* info[0..15]: version, num_types, zbl, zbl_flexible, n_max_r, n_max_a,
 * basis_r, basis_a, L_max, num_L, dim, H, MN_r, MN_a, has_q bitmask
 * (bit0 q222, bit1 q1111, bit2 q112, bit3 q123, bit4 q233, bit5 q134),
 * typewise_zbl.  rc[0..2T-1]: rc_radial[t], rc_angular[t]. */
void nepo_info(const nepo_model* m, int* info, double* rc);

/*
 * The harmonic tables of degrees 1..8: z[9][9][9] the z-polynomial
 * coefficients [L][m][power], c3b[80] the weights of the q_L invariants.
 * Either pointer may be NULL.
 */
void nepo_harmonic_tables(double* z, double* c3b);

/*
 * Per-atom energy, force and virial.
 *   h[9]    box matrix, row-major with the cell vectors a, b, c as columns
 *           (the reference's Box::cpu_h[0..8] layout)
 *   pbc[3]  1 = periodic
 *   pos     3n doubles, SoA (x[n], y[n], z[n])
 *   pe      n doubles; force 3n doubles SoA;
 *   virial  9n doubles SoA, order xx yy zz xy xz yz yx zx zy
 * Outputs are overwritten.  Returns 0 on success.
 */
int nepo_compute(const nepo_model* m, int n, const int* type, const double* h,
                 const int* pbc, const double* pos, double* pe, double* force,
                 double* virial);

/*
 * Descriptor vectors q (already multiplied by q_scaler), dim doubles per atom
 * (atom-major, q[i*dim + d]).
 */
int nepo_descriptors(const nepo_model* m, int n, const int* type, const double* h,
                     const int* pbc, const double* pos, double* q);

/*
 * Typewise neighbour sets of the large-box path with the reference's FP32
 * predicate (double difference rounded to float, float minimum image,
 * float squared distance against the float type-pair cutoff squared).
 * which = 0 radial, 1 angular.  Rows are sorted ascending; row i is
 * nl[i*mn .. i*mn+nn[i]).  Returns 0, or 1 when a row exceeds mn.
 */
int nepo_neighbors_f32(const nepo_model* m, int n, const int* type, const double* h,
                       const int* pbc, const double* pos, int which, int mn, int* nn,
                       int* nl);

#ifdef __cplusplus
}
#endif
#endif
