/*
 * sbd_oracle: CPU restatement of the reference sbd tensor-product-basis
 * selected-CI path (walkup/sbd-ykt), in plain C.
 *
 * TEST INFRASTRUCTURE ONLY. This is the checker the CUDA product is compared
 * against; it is pinned against golden vectors produced by the compiled
 * reference (tests/golden/). Only tests/, __graft_entry__.smoke() and
 * bench.py's CPU-baseline leg may load it. The product never calls it.
 *
 * Conventions (same as the product C-ABI, include/sbdx.h):
 *   - a spin string is one uint64, bit p = spatial orbital p (L <= 64);
 *   - a determinant (ia, ib) has vector index ia*nb + ib (alpha-major);
 *   - h is L*L row-major; eri is the 8-fold packed (pq|rs) array with
 *     index canon(pq, rs), pq = max(p,q)(max(p,q)+1)/2 + min(p,q);
 *   - the interleaved spin-orbital order of the reference is used for all
 *     signs: alpha orbital p -> 2p, beta orbital p -> 2p+1.
 */
#ifndef SBD_ORACLE_H
#define SBD_ORACLE_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

size_t sbo_eri_index(int p, int q, int r, int s);

/* Connectivity of one spin: for each bra string the ascending ket indices at
 * XOR-popcount 2 (singles) and 4 (doubles). idx layout: per bra, singles
 * then doubles. Returns the total entry count; idx may be NULL (count only). */
long long sbo_connectivity(const uint64_t* s, size_t n, uint64_t* slen, uint64_t* dlen, uint64_t* idx);

/* <bra|H|ket> restating Hij (determinants.h:467-526). */
double sbo_hij(int L, double I0, const double* h, const double* eri, uint64_t bra_a, uint64_t bra_b,
               uint64_t ket_a, uint64_t ket_b);

/* Reference parity(det, start, end) on the interleaved determinant of
 * (alpha, beta): returns +1 or -1 (determinants.h:228-279). */
int sbo_parity(uint64_t alpha, uint64_t beta, int start, int end);

void sbo_diag_terms(int L, double I0, const double* h, const double* eri, const uint64_t* a, size_t na,
                    const uint64_t* b, size_t nb, double* hii);

void sbo_sigma(int L, double I0, const double* h, const double* eri, const uint64_t* a, size_t na,
               const uint64_t* b, size_t nb, const double* hii, const double* C, double* S);

/* Off-diagonal part of the bra alpha rows [row0, row0 + rows) of sigma,
 * rows x nb values (the reference mult on a bra block with zero diagonal). */
void sbo_sigma_rows(int L, double I0, const double* h, const double* eri, const uint64_t* a, size_t na,
                    const uint64_t* b, size_t nb, const double* C, size_t row0, size_t rows, double* S);

/* Davidson (davidson.h:661-924) + final <W|HW> (sbdiag.h:250-273).
 * W: in = start vector (NULL -> e_0), out = final normalised vector.
 * Returns the energy; *n_sigma receives the number of sigma products. */
double sbo_davidson(int L, double I0, const double* h, const double* eri, const uint64_t* a, size_t na,
                    const uint64_t* b, size_t nb, int max_it, int max_nb, double eps, double* W,
                    int* n_sigma);

/* 1-/2-RDM restating Correlation (correlation.h:194-444). one: 2*L*L, two: 4*L^4. */
void sbo_rdm(int L, const uint64_t* a, size_t na, const uint64_t* b, size_t nb, const double* W,
             double* one, double* two);

/* OccupationDensity (occupation.h:10-95) over all orbitals: density[2p+s]. */
void sbo_occupation(int L, const uint64_t* a, size_t na, const uint64_t* b, size_t nb, const double* W,
                    double* density);

/* CarryOverAlphaDet (rdmat.h:60-132). ratio == 0 -> threshold rule, else keep
 * (size_t)(ratio*na). order[] receives alpha indices in kept order; returns
 * the kept count; *truncated receives 1 - kept weight (ratio rule). */
long long sbo_carryover(const double* W, size_t na, size_t nb, double ratio, double threshold,
                        uint64_t* order, double* truncated);

/* Energy from RDMs (sample main.cc:166-216): I0 + sum h*g1 + 1/2 sum (ik|jl) G2. */
double sbo_rdm_energy(int L, double I0, const double* h, const double* eri, const double* one,
                      const double* two);

#ifdef __cplusplus
}
#endif
#endif
