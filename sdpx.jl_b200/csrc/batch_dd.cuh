// Float64x2 (double-double) Newton system of the batched engine (included by
// batch.cu inside its kernel namespace).
//
// The iterate (x, X, Y) stays in FP64; the Newton system is formed and solved
// in double-double: the block residuals P = 𝒜x − X − C, d = c − 𝒜ᵀY and
// R = −XY (+μI), X⁻¹ refined from the FP64 inverse by Newton–Schulz steps
// Z ← Z + Z(I − XZ), the Schur matrix S_ij = ⟨A_i, X⁻¹A_jY⟩ (i ≥ j, mirrored),
// its Cholesky factor with the regularisation retries of the FP64 path, the
// right-hand sides, the solves and refinement residuals ρ = r − S·dx, and the
// direction blocks dX = 𝒜dx + P, dY = sym(X⁻¹(R − dX·Y)), rounded to FP64 for
// the step length and the update.  This is the extended-precision setting of
// SDPX (src/kernels/mixed_precision_kkt.jl:1475-1586: a target-precision
// operator and residuals; ext/SDPXMultiFloatLinearAlgebraExt.jl:743-778, the
// Float64x2 provider) for the small instances of a batch, where FP64 stalls
// near a 1e-12 gap because κ(S) passes 1/eps.
//
// Storage: every double-double array is (hi, lo) with hi in the pool's FP64
// array of the same name (a normalised pair's hi is its FP64 rounding, so the
// FP64 kernels keep reading them) and lo in the *l arrays of the pool.
#pragma once

// √a in double-double: one Newton correction of the FP64 root.
__device__ __forceinline__ ddv dd_sqrt(ddv a) {
  const double s = sqrt(a.hi);
  const ddv p = dd_two_prod(s, s);
  const double r = (((a.hi - p.hi) - p.lo) + a.lo) / (2.0 * s);
  return dd_fast_two_sum(s, r);
}
__device__ __forceinline__ ddv dd_fma_d(ddv acc, ddv a, double b) {
  return dd_add(acc, dd_mul_d(a, b));
}
__device__ __forceinline__ ddv dd_warp_sum(ddv v) {
  for (int o = 16; o > 0; o >>= 1) v = dd_add(v, dd_shfl_xor(v, o));
  return v;
}
// Block-wide double-double sum; red holds 64 doubles.
__device__ ddv cta_dd_sum(ddv v, double* red) {
  v = dd_warp_sum(v);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
  __syncthreads();
  if (lane == 0) {
    red[2 * w] = v.hi;
    red[2 * w + 1] = v.lo;
  }
  __syncthreads();
  if (w == 0) {
    ddv t = lane < nw ? ddv{red[2 * lane], red[2 * lane + 1]} : ddv{0.0, 0.0};
    t = dd_warp_sum(t);
    if (lane == 0) {
      red[0] = t.hi;
      red[1] = t.lo;
    }
  }
  __syncthreads();
  const ddv r{red[0], red[1]};
  __syncthreads();
  return r;
}

// D1: P, d and R in double-double (after k_b_residuals factored X and Y);
// kMode 1: only P and d (the solution residuals).  Outputs their FP64 norms.
__global__ void __launch_bounds__(kThreads)
    k_dd_resid(Pool pool, const int* act, const double* par, double* res) {
  INST_PROLOGUE
  extern __shared__ __align__(16) double sm[];
  double* Xs = sm;
  double* Ys = Xs + pool.kq;
  __shared__ double red[32];
  const double* A = pool.A + I.a_off;
  const double* x = pool.x + I.m_off;
  double pmax = 0.0;
  for (long long e = threadIdx.x; e < kk; e += blockDim.x) {
    ddv s{0.0, 0.0};
    for (int j = 0; j < m; ++j) s = dd_add(s, dd_two_prod(x[j], A[(long long)j * kk + e]));
    s = dd_add(s, {-pool.X[I.kk_off + e], 0.0});
    s = dd_add(s, {-pool.C[I.kk_off + e], 0.0});
    dd_store(pool.P + I.kk_off, pool.Pl + I.kk_off, e, s);
    pmax = fmax(pmax, abs_nan_inf(s.hi));
    Xs[e] = pool.X[I.kk_off + e];
    Ys[e] = pool.Y[I.kk_off + e];
  }
  pmax = cta_max(pmax, red);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  double dmax = 0.0;
  for (int j = warp; j < m; j += nw) {
    ddv s{0.0, 0.0};
    for (long long e = lane; e < kk; e += 32) s = dd_add(s, dd_two_prod(A[(long long)j * kk + e], Ys[e]));
    s = dd_warp_sum(s);
    const ddv dv = dd_add({pool.c[I.m_off + j], 0.0}, dd_neg(s));
    if (lane == 0) dd_store(pool.d + I.m_off, pool.dl + I.m_off, j, dv);
    dmax = fmax(dmax, abs_nan_inf(dv.hi));
  }
  dmax = cta_max(dmax, red);
  if (in[kMode] != 1.0) {
    const double mu = in[kMu];
    const bool add_mu = in[kUseAffine] == 0.0;
    for (long long e = threadIdx.x; e < kk; e += blockDim.x) {
      const int r = (int)(e % k), c = (int)(e / k);
      ddv s{0.0, 0.0};
      for (int p = 0; p < k; ++p) s = dd_add(s, dd_two_prod(Xs[r + p * k], Ys[p + c * k]));
      s = dd_neg(s);
      if (add_mu && r == c) s = dd_add(s, {mu, 0.0});
      dd_store(pool.R + I.kk_off, pool.Rl + I.kk_off, e, s);
    }
  }
  if (threadIdx.x == 0) {
    out[oPres] = pmax;
    out[oDres] = dmax;
  }
}

// D2: X⁻¹ in double-double from the FP64 factor's W = L_X⁻¹: Z = WᵀW
// (symmetrised), then three Newton–Schulz steps Z ← sym(Z + Z(I − XZ)).
__global__ void __launch_bounds__(kThreads)
    k_dd_xinv(Pool pool, const int* act, const double* par, double* res) {
  INST_PROLOGUE
  extern __shared__ __align__(16) double sm[];
  double* Xs = sm;
  double* Zh = Xs + pool.kq;
  double* Zl = Zh + pool.kq;
  double* Mh = Zl + pool.kq;
  double* Ml = Mh + pool.kq;
  const double* W = pool.W + I.kk_off;
  double* Xih = pool.Xih + I.kk_off;
  double* Xil = pool.Xil + I.kk_off;
  for (long long e = threadIdx.x; e < kk; e += blockDim.x) {
    Xs[e] = pool.X[I.kk_off + e];
    Mh[e] = W[e];
  }
  __syncthreads();
  for (long long e = threadIdx.x; e < kk; e += blockDim.x) {  // Z0 = WᵀW (W lower)
    const int r = (int)(e % k), c = (int)(e / k);
    double s = 0.0;
    for (int p = max(r, c); p < k; ++p) s += Mh[p + r * k] * Mh[p + c * k];
    Zh[e] = s;
  }
  __syncthreads();
  for (long long e = threadIdx.x; e < kk; e += blockDim.x) {
    const int r = (int)(e % k), c = (int)(e / k);
    Ml[e] = 0.5 * (Zh[e] + Zh[c + r * k]);
  }
  __syncthreads();
  for (long long e = threadIdx.x; e < kk; e += blockDim.x) {
    Zh[e] = Ml[e];
    Zl[e] = 0.0;
  }
  __syncthreads();
  for (int step = 0; step < 3; ++step) {
    for (long long e = threadIdx.x; e < kk; e += blockDim.x) {  // M = I − X·Z
      const int r = (int)(e % k), c = (int)(e / k);
      ddv s{r == c ? 1.0 : 0.0, 0.0};
      for (int p = 0; p < k; ++p) s = dd_add(s, dd_neg(dd_mul_d({Zh[p + c * k], Zl[p + c * k]}, Xs[r + p * k])));
      Mh[e] = s.hi;
      Ml[e] = s.lo;
    }
    __syncthreads();
    for (long long e = threadIdx.x; e < kk; e += blockDim.x) {  // Z + Z·M → global
      const int r = (int)(e % k), c = (int)(e / k);
      ddv s{Zh[e], Zl[e]};
      for (int p = 0; p < k; ++p)
        s = dd_add(s, dd_mul({Zh[r + p * k], Zl[r + p * k]}, {Mh[p + c * k], Ml[p + c * k]}));
      Xih[e] = s.hi;
      Xil[e] = s.lo;
    }
    __syncthreads();
    for (long long e = threadIdx.x; e < kk; e += blockDim.x) {  // symmetrise back into Z
      const int r = (int)(e % k), c = (int)(e / k);
      const long long t = c + (long long)r * k;
      const ddv a{Xih[e], Xil[e]}, b{Xih[t], Xil[t]};
      const ddv s = dd_mul_d(dd_add(a, b), 0.5);
      Zh[e] = s.hi;
      Zl[e] = s.lo;
    }
    __syncthreads();
  }
  for (long long e = threadIdx.x; e < kk; e += blockDim.x) {
    Xih[e] = Zh[e];
    Xil[e] = Zl[e];
  }
}

// D3: the Schur columns j ∈ [lo, hi) of one work item: G_j = X⁻¹·A_j·Y
// (double-double X⁻¹, FP64 A_j and Y) into the panel, then the lower part
// S(i, j) = ⟨A_i, G_j⟩, i ≥ j (one warp per i); k_dd_factor mirrors it.
__global__ void k_dd_schur(Pool pool, const int* act, const int4* work) {
  const int4 wi = work[blockIdx.x];
  const Inst I = pool.inst[act[wi.x]];
  const int k = I.k, m = I.m;
  const long long kk = (long long)k * k;
  extern __shared__ __align__(16) double sm[];
  double* Zh = sm;
  double* Zl = Zh + pool.kq;
  double* As = Zl + pool.kq;
  double* Th = As + pool.kq;
  double* Tl = Th + pool.kq;
  for (long long e = threadIdx.x; e < kk; e += blockDim.x) {
    Zh[e] = pool.Xih[I.kk_off + e];
    Zl[e] = pool.Xil[I.kk_off + e];
  }
  const double* A = pool.A + I.a_off;
  const double* Y = pool.Y + I.kk_off;
  double* Gh = pool.Ph + I.a_off;
  double* Gl = pool.Gl + I.a_off;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  for (int j = wi.y; j < wi.z; ++j) {
    for (long long e = threadIdx.x; e < kk; e += blockDim.x) As[e] = A[(long long)j * kk + e];
    __syncthreads();
    for (long long e = threadIdx.x; e < kk; e += blockDim.x) {  // T = X⁻¹·A_j
      const int r = (int)(e % k), c = (int)(e / k);
      ddv s{0.0, 0.0};
      for (int p = 0; p < k; ++p) s = dd_fma_d(s, {Zh[r + p * k], Zl[r + p * k]}, As[p + c * k]);
      Th[e] = s.hi;
      Tl[e] = s.lo;
    }
    __syncthreads();
    for (long long e = threadIdx.x; e < kk; e += blockDim.x) {  // G_j = T·Y
      const int r = (int)(e % k), c = (int)(e / k);
      ddv s{0.0, 0.0};
      for (int p = 0; p < k; ++p) s = dd_fma_d(s, {Th[r + p * k], Tl[r + p * k]}, Y[p + c * k]);
      Gh[(long long)j * kk + e] = s.hi;
      Gl[(long long)j * kk + e] = s.lo;
    }
    __syncthreads();
    for (int i = j + warp; i < m; i += nw) {  // S(i, j) = ⟨A_i, G_j⟩, i ≥ j
      ddv s{0.0, 0.0};
      for (long long e = lane; e < kk; e += 32)
        s = dd_fma_d(s, {Gh[(long long)j * kk + e], Gl[(long long)j * kk + e]},
                     A[(long long)i * kk + e]);
      s = dd_warp_sum(s);
      if (lane == 0) dd_store(pool.S + I.mm_off, pool.Sl + I.mm_off, i + (long long)j * m, s);
    }
    __syncthreads();
  }
}

// D4: S's upper triangle ← its lower one, then the double-double Cholesky of S with ≤ 6
// regularisation retries S_ii += δ·max(|S_ii|, 1), δ = √eps then ×10 (as the
// FP64 path, src/kkt.jl:1419-1445); quality = min/max |L_jj|.
__global__ void __launch_bounds__(kThreads)
    k_dd_factor(Pool pool, const int* act, const double* par, double* res) {
  INST_PROLOGUE
  __shared__ double sflag[4];
  double* Sh = pool.S + I.mm_off;
  double* Sl = pool.Sl + I.mm_off;
  double* Lh = pool.LS + I.mm_off;
  double* Ll = pool.LSl + I.mm_off;
  const long long mm = (long long)m * m;
  for (long long e = threadIdx.x; e < mm; e += blockDim.x) {  // upper ← lower
    const int r = (int)(e % m), c = (int)(e / m);
    if (r < c) {
      const long long t = c + (long long)r * m;
      Sh[e] = Sh[t];
      Sl[e] = Sl[t];
    }
  }
  __syncthreads();
  int attempts = 0;
  double reg = 0.0;
  bool ok = false;
  while (true) {
    for (long long e = threadIdx.x; e < mm; e += blockDim.x) {
      const int r = (int)(e % m), c = (int)(e / m);
      ddv v = r >= c ? ddv{Sh[e], Sl[e]} : ddv{0.0, 0.0};
      if (r == c && attempts > 0) v = dd_add(v, {reg * fmax(fabs(Sh[e]), 1.0), 0.0});
      Lh[e] = v.hi;
      Ll[e] = v.lo;
    }
    __syncthreads();
    ok = true;
    for (int j = 0; j < m; ++j) {
      if (threadIdx.x == 0) {
        const ddv d{Lh[j + (long long)j * m], Ll[j + (long long)j * m]};
        sflag[0] = d.hi > 0.0 ? 1.0 : 0.0;
        if (d.hi > 0.0) {
          const ddv s = dd_sqrt(d);
          sflag[1] = s.hi;
          sflag[2] = s.lo;
        }
      }
      __syncthreads();
      if (sflag[0] == 0.0) {
        ok = false;
        break;
      }
      const ddv ljj{sflag[1], sflag[2]};
      for (int i = j + 1 + threadIdx.x; i < m; i += blockDim.x) {
        const long long e = i + (long long)j * m;
        const ddv q = dd_div({Lh[e], Ll[e]}, ljj);
        Lh[e] = q.hi;
        Ll[e] = q.lo;
      }
      if (threadIdx.x == 0) {
        Lh[j + (long long)j * m] = ljj.hi;
        Ll[j + (long long)j * m] = ljj.lo;
      }
      __syncthreads();
      const int rem = m - j - 1;
      for (long long e = threadIdx.x; e < (long long)rem * rem; e += blockDim.x) {
        const int ii = j + 1 + (int)(e % rem), ll = j + 1 + (int)(e / rem);
        if (ii >= ll) {
          const long long t = ii + (long long)ll * m;
          const long long a = ii + (long long)j * m, b = ll + (long long)j * m;
          const ddv v = dd_add({Lh[t], Ll[t]}, dd_neg(dd_mul({Lh[a], Ll[a]}, {Lh[b], Ll[b]})));
          Lh[t] = v.hi;
          Ll[t] = v.lo;
        }
      }
      __syncthreads();
    }
    __syncthreads();
    if (ok || attempts >= 6) break;
    ++attempts;
    reg = attempts == 1 ? 1.4901161193847656e-08 : reg * 10.0;
  }
  if (threadIdx.x == 0) {
    out[oOk] = ok ? 1.0 : 0.0;
    out[oReg] = attempts;
    double q = 0.0;
    if (ok) {
      double mn = fabs(Lh[0]), mx = mn;
      for (int j = 1; j < m; ++j) {
        mn = fmin(mn, fabs(Lh[j + (long long)j * m]));
        mx = fmax(mx, fabs(Lh[j + (long long)j * m]));
      }
      q = (mx > 0 && isfinite(mx)) ? fmin(1.0, fmax(0.0, mn / mx)) : 0.0;
    }
    out[oQual] = q;
  }
}

// D5: kMode 0: dx = S⁻¹r; kMode 1: dxb = dx, dx += S⁻¹ρ — in double-double
// with the double-double factor.
__global__ void __launch_bounds__(kThreads)
    k_dd_solve(Pool pool, const int* act, const double* par, double* res) {
  INST_PROLOGUE
  __shared__ double vh[kMaxM], vl[kMaxM];
  __shared__ double red[64];
  const bool corr = in[kMode] == 1.0;
  const double* sh = corr ? pool.rho + I.m_off : pool.r + I.m_off;
  const double* sl = corr ? pool.rhol + I.m_off : pool.rl + I.m_off;
  const double* Lh = pool.LS + I.mm_off;
  const double* Ll = pool.LSl + I.mm_off;
  for (int i = threadIdx.x; i < m; i += blockDim.x) {
    vh[i] = sh[i];
    vl[i] = sl[i];
  }
  for (int j = 0; j < m; ++j) {  // forward
    __syncthreads();
    const long long djj = j + (long long)j * m;
    const ddv yj = dd_div({vh[j], vl[j]}, {Lh[djj], Ll[djj]});
    __syncthreads();
    if (threadIdx.x == 0) {
      vh[j] = yj.hi;
      vl[j] = yj.lo;
    }
    for (int i = j + 1 + threadIdx.x; i < m; i += blockDim.x) {
      const long long e = i + (long long)j * m;
      const ddv v = dd_add({vh[i], vl[i]}, dd_neg(dd_mul({Lh[e], Ll[e]}, yj)));
      vh[i] = v.hi;
      vl[i] = v.lo;
    }
  }
  for (int j = m - 1; j >= 0; --j) {  // backward
    __syncthreads();
    ddv s{0.0, 0.0};
    for (int i = j + 1 + threadIdx.x; i < m; i += blockDim.x) {
      const long long e = i + (long long)j * m;
      s = dd_add(s, dd_mul({Lh[e], Ll[e]}, {vh[i], vl[i]}));
    }
    s = cta_dd_sum(s, red);
    if (threadIdx.x == 0) {
      const long long djj = j + (long long)j * m;
      const ddv v = dd_div(dd_add({vh[j], vl[j]}, dd_neg(s)), {Lh[djj], Ll[djj]});
      vh[j] = v.hi;
      vl[j] = v.lo;
    }
  }
  __syncthreads();
  double* dxh = pool.dx + I.m_off;
  double* dxl = pool.dxl + I.m_off;
  for (int i = threadIdx.x; i < m; i += blockDim.x) {
    if (corr) {
      pool.dxb[I.m_off + i] = dxh[i];
      pool.dxbl[I.m_off + i] = dxl[i];
      const ddv v = dd_add({dxh[i], dxl[i]}, {vh[i], vl[i]});
      dxh[i] = v.hi;
      dxl[i] = v.lo;
    } else {
      dxh[i] = vh[i];
      dxl[i] = vl[i];
    }
  }
}

// D6: r = −(d + 𝒜ᵀ vec(X⁻¹(P·Y − R))) in double-double; kMode 1 first forms
// the corrector R = kTarget·I − X·Y − dX·dY (FP64 dX, dY).
__global__ void __launch_bounds__(kThreads)
    k_dd_rhs(Pool pool, const int* act, const double* par, double* res) {
  INST_PROLOGUE
  extern __shared__ __align__(16) double sm[];
  double* Ys = sm;
  double* Zh = Ys + pool.kq;
  double* Zl = Zh + pool.kq;
  double* Xh = Zl + pool.kq;
  double* Xl = Xh + pool.kq;
  double* Rh = pool.R + I.kk_off;
  double* Rl = pool.Rl + I.kk_off;
  for (long long e = threadIdx.x; e < kk; e += blockDim.x) {
    Ys[e] = pool.Y[I.kk_off + e];
    Xh[e] = pool.X[I.kk_off + e];
  }
  __syncthreads();
  if (in[kMode] == 1.0) {
    const double* dX = pool.dX + I.kk_off;
    const double* dY = pool.dY + I.kk_off;
    for (long long e = threadIdx.x; e < kk; e += blockDim.x) {
      const int r = (int)(e % k), c = (int)(e / k);
      ddv s{0.0, 0.0};
      for (int p = 0; p < k; ++p) {
        s = dd_add(s, dd_two_prod(Xh[r + p * k], Ys[p + c * k]));
        s = dd_add(s, dd_two_prod(dX[r + p * k], dY[p + c * k]));
      }
      s = dd_neg(s);
      if (r == c) s = dd_add(s, {in[kTarget], 0.0});
      Rh[e] = s.hi;
      Rl[e] = s.lo;
    }
    __syncthreads();
  }
  const double* Ph = pool.P + I.kk_off;
  const double* Pl = pool.Pl + I.kk_off;
  for (long long e = threadIdx.x; e < kk; e += blockDim.x) {  // Z = P·Y − R
    const int r = (int)(e % k), c = (int)(e / k);
    ddv s = dd_neg({Rh[e], Rl[e]});
    for (int p = 0; p < k; ++p) s = dd_fma_d(s, {Ph[r + p * k], Pl[r + p * k]}, Ys[p + c * k]);
    Zh[e] = s.hi;
    Zl[e] = s.lo;
  }
  __syncthreads();
  for (long long e = threadIdx.x; e < kk; e += blockDim.x) {
    Xh[e] = pool.Xih[I.kk_off + e];
    Xl[e] = pool.Xil[I.kk_off + e];
  }
  __syncthreads();
  double* Wh = pool.Z + I.kk_off;
  double* Wl = pool.Zl + I.kk_off;
  for (long long e = threadIdx.x; e < kk; e += blockDim.x) {  // X⁻¹·Z
    const int r = (int)(e % k), c = (int)(e / k);
    ddv s{0.0, 0.0};
    for (int p = 0; p < k; ++p)
      s = dd_add(s, dd_mul({Xh[r + p * k], Xl[r + p * k]}, {Zh[p + c * k], Zl[p + c * k]}));
    Wh[e] = s.hi;
    Wl[e] = s.lo;
  }
  __syncthreads();
  const double* A = pool.A + I.a_off;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  for (int j = warp; j < m; j += nw) {
    ddv s{0.0, 0.0};
    for (long long e = lane; e < kk; e += 32) s = dd_fma_d(s, {Wh[e], Wl[e]}, A[(long long)j * kk + e]);
    s = dd_warp_sum(s);
    if (lane == 0) {
      const ddv v = dd_neg(dd_add({pool.d[I.m_off + j], pool.dl[I.m_off + j]}, s));
      pool.r[I.m_off + j] = v.hi;
      pool.rl[I.m_off + j] = v.lo;
    }
  }
}

// D7: dX = 𝒜dx + P and dY = sym(X⁻¹(R − dX·Y)) in double-double, stored
// rounded to FP64 (pool.dX, pool.dY).
__global__ void __launch_bounds__(kThreads)
    k_dd_dirblocks(Pool pool, const int* act, const double* par, double* res) {
  INST_PROLOGUE
  extern __shared__ __align__(16) double sm[];
  double* Dh = sm;  // dX, then X⁻¹
  double* Dl = Dh + pool.kq;
  double* Ys = Dl + pool.kq;
  double* Th = Ys + pool.kq;
  double* Tl = Th + pool.kq;
  const double* A = pool.A + I.a_off;
  const double* dxh = pool.dx + I.m_off;
  const double* dxl = pool.dxl + I.m_off;
  for (long long e = threadIdx.x; e < kk; e += blockDim.x) {
    ddv s{pool.P[I.kk_off + e], pool.Pl[I.kk_off + e]};
    for (int j = 0; j < m; ++j) s = dd_fma_d(s, {dxh[j], dxl[j]}, A[(long long)j * kk + e]);
    Dh[e] = s.hi;
    Dl[e] = s.lo;
    pool.dX[I.kk_off + e] = s.hi;
    Ys[e] = pool.Y[I.kk_off + e];
  }
  __syncthreads();
  for (long long e = threadIdx.x; e < kk; e += blockDim.x) {  // T = R − dX·Y
    const int r = (int)(e % k), c = (int)(e / k);
    ddv s{pool.R[I.kk_off + e], pool.Rl[I.kk_off + e]};
    for (int p = 0; p < k; ++p) s = dd_add(s, dd_neg(dd_mul_d({Dh[r + p * k], Dl[r + p * k]}, Ys[p + c * k])));
    Th[e] = s.hi;
    Tl[e] = s.lo;
  }
  __syncthreads();
  for (long long e = threadIdx.x; e < kk; e += blockDim.x) {
    Dh[e] = pool.Xih[I.kk_off + e];
    Dl[e] = pool.Xil[I.kk_off + e];
  }
  __syncthreads();
  double* Wh = pool.Z + I.kk_off;
  double* Wl = pool.Zl + I.kk_off;
  for (long long e = threadIdx.x; e < kk; e += blockDim.x) {  // X⁻¹·T
    const int r = (int)(e % k), c = (int)(e / k);
    ddv s{0.0, 0.0};
    for (int p = 0; p < k; ++p)
      s = dd_add(s, dd_mul({Dh[r + p * k], Dl[r + p * k]}, {Th[p + c * k], Tl[p + c * k]}));
    Wh[e] = s.hi;
    Wl[e] = s.lo;
  }
  __syncthreads();
  for (long long e = threadIdx.x; e < kk; e += blockDim.x) {
    const int r = (int)(e % k), c = (int)(e / k);
    const long long t = c + (long long)r * k;
    pool.dY[I.kk_off + e] = dd_mul_d(dd_add({Wh[e], Wl[e]}, {Wh[t], Wl[t]}), 0.5).hi;
  }
}

// D8: ρ = r − S·dx in double-double (S symmetric, stored full); ‖ρ‖∞, ‖r‖∞.
__global__ void __launch_bounds__(kThreads)
    k_dd_rho(Pool pool, const int* act, const double* par, double* res) {
  INST_PROLOGUE
  __shared__ double red[32];
  const double* Sh = pool.S + I.mm_off;
  const double* Sl = pool.Sl + I.mm_off;
  const double* dxh = pool.dx + I.m_off;
  const double* dxl = pool.dxl + I.m_off;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  double rm = 0.0, rn = 0.0;
  for (int i = warp; i < m; i += nw) {
    ddv s{0.0, 0.0};
    for (int j = lane; j < m; j += 32) {
      const long long e = j + (long long)i * m;
      s = dd_add(s, dd_mul({Sh[e], Sl[e]}, {dxh[j], dxl[j]}));
    }
    s = dd_warp_sum(s);
    const ddv v = dd_add({pool.r[I.m_off + i], pool.rl[I.m_off + i]}, dd_neg(s));
    if (lane == 0) {
      pool.rho[I.m_off + i] = v.hi;
      pool.rhol[I.m_off + i] = v.lo;
    }
    rm = fmax(rm, abs_nan_inf(v.hi));
    rn = fmax(rn, abs_nan_inf(pool.r[I.m_off + i]));
  }
  rm = cta_max(rm, red);
  rn = cta_max(rn, red);
  if (threadIdx.x == 0) {
    out[oRes] = rm;
    out[oRnorm] = rn;
  }
}

// D9: dx ← dxb in double-double (a correction that did not reduce ρ).
__global__ void k_dd_rollback(Pool pool, const int* act, const double* par, double* res) {
  INST_PROLOGUE
  for (int i = threadIdx.x; i < m; i += blockDim.x) {
    pool.dx[I.m_off + i] = pool.dxb[I.m_off + i];
    pool.dxl[I.m_off + i] = pool.dxbl[I.m_off + i];
  }
}
