/*
 * ORACLE -- test infrastructure, not product code.  See oracle_kernels.h.
 *
 * Plain-C restatement of the Monalisa reference kernels.  The arithmetic
 * order (loops over points, then window z/y/x, then channels; per-row nnz in
 * stored order) is kept identical to the reference so that, compiled without
 * FMA contraction, the results match the compiled reference bit for bit.
 * The code itself is written independently: window cells are enumerated by
 * integer offsets and the jump-coded indices are decoded into absolute
 * positions rather than walked with running pointers.
 */
#include "oracle_kernels.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

/* Window geometry shared by every leight kernel
 * (bmGridder_n2u_leight3_mex.cpp:189-199): odd widths centre the window on
 * the nearest node (shift 0.5), even widths start at floor(t). */
static void window_geometry(int nWin, float* t_shift, int* half) {
  if (nWin % 2) {
    *t_shift = 0.5f;
    *half = (nWin - 1) / 2;
  } else {
    *t_shift = 0.0f;
    *half = nWin / 2 - 1;
  }
}

void oracle_gridder_leight(int imDim, const float* aReal, const float* aImag,
                           const float* tx, const float* ty, const float* tz,
                           const float* Dn, int nCh, int nPt, int Nx, int Ny,
                           int Nz, int nWin, float kernelParam_1,
                           float kernelParam_2, float* bReal, float* bImag) {
  (void)kernelParam_2; /* the reference ignores it (K_max is deapodisation-only) */
  const int dims[3] = {Nx, imDim > 1 ? Ny : 1, imDim > 2 ? Nz : 1};
  const long long nCells = (long long)dims[0] * dims[1] * dims[2];
  const long long strideY = dims[0], strideZ = (long long)dims[0] * dims[1];

  float t_shift;
  int half;
  window_geometry(nWin, &t_shift, &half);

  /* Gaussian constants exactly as leight3_mex.cpp:202-205 computes them */
  const float sigma = kernelParam_1;
  const float g1 = 1 / ((float)sqrt(2 * 3.141592) * sigma);
  const float g2 = -1 / (2 * (sigma * sigma));

  float* norm = (float*)calloc((size_t)nCells, sizeof(float));
  memset(bReal, 0, sizeof(float) * (size_t)nCells * (size_t)nCh);
  memset(bImag, 0, sizeof(float) * (size_t)nCells * (size_t)nCh);

  const int wz = imDim > 2 ? nWin : 1;
  const int wy = imDim > 1 ? nWin : 1;

  for (int p = 0; p < nPt; ++p) {
    float t[3] = {tx[p], imDim > 1 ? ty[p] : 0.f, imDim > 2 ? tz[p] : 0.f};
    float r[3];
    int c[3];
    for (int d = 0; d < 3; ++d) {
      float node;
      modff(t[d] + t_shift, &node);
      r[d] = t[d] - node;
      c[d] = (int)node - 1; /* 0-based centre cell */
    }
    const float dn = Dn[p];
    const float* ar = aReal + (long long)p * nCh;
    const float* ai = aImag + (long long)p * nCh;

    for (int iz = 0; iz < wz; ++iz) {
      const int nz = imDim > 2 ? c[2] - half + iz : 0;
      const float uz = imDim > 2 ? (float)(iz - half) : 0.f;
      if (nz < 0 || nz > dims[2] - 1) continue;
      for (int iy = 0; iy < wy; ++iy) {
        const int ny = imDim > 1 ? c[1] - half + iy : 0;
        const float uy = imDim > 1 ? (float)(iy - half) : 0.f;
        if (ny < 0 || ny > dims[1] - 1) continue;
        for (int ix = 0; ix < nWin; ++ix) {
          const int nx = c[0] - half + ix;
          const float ux = (float)(ix - half);
          if (nx < 0 || nx > dims[0] - 1) continue;
          /* squared distance summed in x, y, z order like the reference */
          const float dx = r[0] - ux;
          float d2 = dx * dx;
          if (imDim > 1) {
            const float dy = r[1] - uy;
            d2 = d2 + dy * dy;
          }
          if (imDim > 2) {
            const float dz = r[2] - uz;
            d2 = d2 + dz * dz;
          }
          const float w = g1 * expf(g2 * d2) * dn;
          const long long cell = nx + ny * strideY + nz * strideZ;
          norm[cell] += w;
          float* br = bReal + cell * nCh;
          float* bi = bImag + cell * nCh;
          for (int k = 0; k < nCh; ++k) {
            br[k] += w * ar[k];
            bi[k] += w * ai[k];
          }
        }
      }
    }
  }

  for (long long cell = 0; cell < nCells; ++cell) {
    float s = norm[cell];
    if (s < 1e-5) s = 1.0f; /* leight3_mex.cpp:341 */
    for (int k = 0; k < nCh; ++k) {
      bReal[cell * nCh + k] /= s;
      bImag[cell * nCh + k] /= s;
    }
  }
  free(norm);
}

void oracle_gridder_n2u(const float* aReal, const float* aImag, const float* w,
                        const int* nJump, int nNb, int nCh, int nPt,
                        int Nu_tot, float* bReal, float* bImag) {
  float* norm = (float*)calloc((size_t)Nu_tot, sizeof(float));
  memset(bReal, 0, sizeof(float) * (size_t)Nu_tot * (size_t)nCh);
  memset(bImag, 0, sizeof(float) * (size_t)Nu_tot * (size_t)nCh);
  long long cell = 0; /* jump-decoded absolute target cell */
  for (int p = 0; p < nPt; ++p) {
    const float* ar = aReal + (long long)p * nCh;
    const float* ai = aImag + (long long)p * nCh;
    for (int j = 0; j < nNb; ++j) {
      const long long e = (long long)p * nNb + j;
      cell += nJump[e];
      const float wt = w[e];
      norm[cell] += wt;
      for (int k = 0; k < nCh; ++k) {
        bReal[cell * nCh + k] += wt * ar[k];
        bImag[cell * nCh + k] += wt * ai[k];
      }
    }
  }
  for (long long c = 0; c < Nu_tot; ++c) {
    float s = norm[c];
    if (s < 1e-5) s = 1.0f; /* bmGridder_n2u_mex.cpp:181-184 */
    for (int k = 0; k < nCh; ++k) {
      bReal[c * nCh + k] /= s;
      bImag[c * nCh + k] /= s;
    }
  }
  free(norm);
}

/* Decodes one matrix's jump arrays into absolute 0-based columns and output
 * rows.  The first r_jump / l_jump entry is absolute, the rest are deltas
 * (bmSparseMat.m:135-166). */
static void decode_jumps(int l_nJump, const int* r_nJump, const int* r_jump,
                         const int* l_jump, long long** cols_out,
                         long long** rows_out, long long* nnz_out) {
  long long nnz = 0;
  for (int i = 0; i < l_nJump; ++i) nnz += r_nJump[i];
  long long* cols = (long long*)malloc(sizeof(long long) * (size_t)(nnz ? nnz : 1));
  long long* rows = (long long*)malloc(sizeof(long long) * (size_t)(l_nJump ? l_nJump : 1));
  long long col = 0, row = 0;
  for (long long e = 0; e < nnz; ++e) {
    col += r_jump[e];
    cols[e] = col;
  }
  for (int i = 0; i < l_nJump; ++i) {
    if (l_jump) {
      row += l_jump[i];
      rows[i] = row;
    } else {
      rows[i] = i;
    }
  }
  *cols_out = cols;
  *rows_out = rows;
  *nnz_out = nnz;
}

void oracle_spmv_cC(int r_size, const int* r_jump, const int* r_nJump,
                    const float* m_val, int l_size, const int* l_jump,
                    int l_nJump, const float* vReal, const float* vImag,
                    int nVec, float* wReal, float* wImag) {
  long long *cols, *rows, nnz;
  decode_jumps(l_nJump, r_nJump, r_jump, l_jump, &cols, &rows, &nnz);
  /* one (vector, real|imag) pair per task, like the OpenMP reference */
#pragma omp parallel for schedule(static)
  for (int task = 0; task < 2 * nVec; ++task) {
    const int k = task / 2;
    const float* v = (task % 2 ? vImag : vReal) + (long long)r_size * k;
    float* w = (task % 2 ? wImag : wReal) + (long long)l_size * k;
    memset(w, 0, sizeof(float) * (size_t)l_size);
    long long e = 0;
    for (int i = 0; i < l_nJump; ++i) {
      float acc = w[rows[i]];
      for (int j = 0; j < r_nJump[i]; ++j, ++e) acc += m_val[e] * v[cols[e]];
      w[rows[i]] = acc;
    }
  }
  (void)nnz;
  free(cols);
  free(rows);
}

void oracle_spmv_cR(int r_size, const int* r_jump, const int* r_nJump,
                    const float* m_val, int l_size, const int* l_jump,
                    int l_nJump, const float* vReal, const float* vImag,
                    int nVec, float* wReal, float* wImag) {
  (void)r_size;
  long long *cols, *rows, nnz;
  decode_jumps(l_nJump, r_nJump, r_jump, l_jump, &cols, &rows, &nnz);
  memset(wReal, 0, sizeof(float) * (size_t)l_size * (size_t)nVec);
  memset(wImag, 0, sizeof(float) * (size_t)l_size * (size_t)nVec);
  long long e0 = 0;
  for (int i = 0; i < l_nJump; ++i) {
    float* wr = wReal + rows[i] * nVec;
    float* wi = wImag + rows[i] * nVec;
    for (int k = 0; k < nVec; ++k) {
      float sr = 0.f, si = 0.f;
      for (int j = 0; j < r_nJump[i]; ++j) {
        const long long e = e0 + j;
        sr += vReal[cols[e] * nVec + k] * m_val[e];
        si += vImag[cols[e] * nVec + k] * m_val[e];
      }
      wr[k] = sr;
      wi[k] = si;
    }
    e0 += r_nJump[i];
  }
  (void)nnz;
  free(cols);
  free(rows);
}

void oracle_spmv_rC(int r_size, const int* r_jump, const int* r_nJump,
                    const float* m_val, int l_size, const int* l_jump,
                    int l_nJump, const float* v, int nVec, float* w) {
  long long *cols, *rows, nnz;
  decode_jumps(l_nJump, r_nJump, r_jump, l_jump, &cols, &rows, &nnz);
  memset(w, 0, sizeof(float) * (size_t)l_size * (size_t)nVec);
  for (int k = 0; k < nVec; ++k) {
    const float* vk = v + (long long)r_size * k;
    float* wk = w + (long long)l_size * k;
    long long e = 0;
    for (int i = 0; i < l_nJump; ++i) {
      float acc = wk[rows[i]];
      for (int j = 0; j < r_nJump[i]; ++j, ++e) acc += m_val[e] * vk[cols[e]];
      wk[rows[i]] = acc;
    }
  }
  (void)nnz;
  free(cols);
  free(rows);
}

long long oracle_r_nJump2index(const int* r_nJump, int l_nJump, int* out) {
  long long n = 0;
  for (int i = 0; i < l_nJump; ++i)
    for (int j = 0; j < r_nJump[i]; ++j) out[n++] = i;
  return n;
}
