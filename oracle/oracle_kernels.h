/*
 * ORACLE -- test infrastructure, not product code.
 *
 * Plain-C restatement of the Monalisa reference's native gridding and
 * sparse-matrix kernels.  Used only by tests/, by __graft_entry__.smoke() and
 * by bench.py's CPU-baseline leg, as the checker for the CUDA library.  It is
 * itself pinned against the reference's own C++ kernels compiled from source
 * (oracle/_ref, built by `make ref`) and against the golden fixtures in
 * tests/golden/, which were produced by those compiled reference kernels.
 *
 * Every function follows the reference's arithmetic order (same loop nesting,
 * same float operations, no FMA contraction) so results are bit-identical to
 * the compiled reference kernels on the same inputs.
 */
#ifndef MLG_ORACLE_KERNELS_H
#define MLG_ORACLE_KERNELS_H

#ifdef __cplusplus
extern "C" {
#endif

/* Adjoint gridding with an on-the-fly Gaussian window, clipped at the grid
 * border and normalised per cell.  imDim = 1, 2 or 3 (ty/tz unused below it).
 * Follows src/gridding123/mex/bmGridder_n2u_leight{1,2,3}/..._mex.cpp
 * (leight3: lines 116-358).  a*: [nCh, nPt] (channel fastest); t*: 1-based
 * grid coordinates; out b*: [nCh, Nx*Ny*Nz]. */
void oracle_gridder_leight(int imDim, const float* aReal, const float* aImag,
                           const float* tx, const float* ty, const float* tz,
                           const float* Dn, int nCh, int nPt, int Nx, int Ny,
                           int Nz, int nWin, float kernelParam_1,
                           float kernelParam_2, float* bReal, float* bImag);

/* Adjoint gridding with precomputed weights w[nNb*nPt] and jump-coded target
 * cells nJump[nNb*nPt] (first jump absolute), normalised per cell.
 * Follows src/gridding123/mex/bmGridder_n2u/bmGridder_n2u_mex.cpp:72-201. */
void oracle_gridder_n2u(const float* aReal, const float* aImag, const float* w,
                        const int* nJump, int nNb, int nCh, int nPt,
                        int Nu_tot, float* bReal, float* bImag);

/* w[:,k] = M v[:,k] over the jump-coded CSR (column layout: v[r_size, nVec],
 * w[l_size, nVec]).  l_jump == NULL means no row squeezing.
 * Follows bmSparseMat_cC_oBlock(_omp)_mex.cpp (omp: lines 106-260). */
void oracle_spmv_cC(int r_size, const int* r_jump, const int* r_nJump,
                    const float* m_val, int l_size, const int* l_jump,
                    int l_nJump, const float* vReal, const float* vImag,
                    int nVec, float* wReal, float* wImag);

/* Same product in row layout (v[nVec, r_size], w[nVec, l_size]).
 * Follows bmSparseMat_cR_oBlock_mex.cpp:82-223. */
void oracle_spmv_cR(int r_size, const int* r_jump, const int* r_nJump,
                    const float* m_val, int l_size, const int* l_jump,
                    int l_nJump, const float* vReal, const float* vImag,
                    int nVec, float* wReal, float* wImag);

/* Real-valued column-layout product (bmSparseMat_rC_oBlock_mex.cpp). */
void oracle_spmv_rC(int r_size, const int* r_jump, const int* r_nJump,
                    const float* m_val, int l_size, const int* l_jump,
                    int l_nJump, const float* v, int nVec, float* w);

/* Expands per-row counts to 1-based row indices
 * (bmSparseMat_r_nJump2index_mex.cpp:70-80).  Returns the number written. */
long long oracle_r_nJump2index(const int* r_nJump, int l_nJump, int* out);

#ifdef __cplusplus
}
#endif
#endif
