// fft_impl.cuh -- the transform kernels of fft.cu, written once over the
// scalar type `real` (with `real2` its complex pair and mk2 its constructor)
// and included by fft.cu into one namespace per precision: FP64 for the plain
// path, FP32 for the mixed-precision form.  Not a standalone header.
__device__ __forceinline__ real2 cmul(real2 a, real2 b) {
  return mk2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ real2 cadd(real2 a, real2 b) { return mk2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ real2 csub(real2 a, real2 b) { return mk2(a.x - b.x, a.y - b.y); }

// forward DFT of size R in registers (exp(-2 pi i rt/R))
template <int R>
__device__ __forceinline__ void small_dft(real2* a) {
  if (R == 2) {
    real2 t0 = cadd(a[0], a[1]), t1 = csub(a[0], a[1]);
    a[0] = t0; a[1] = t1;
  } else if (R == 4) {
    real2 t0 = cadd(a[0], a[2]), t1 = csub(a[0], a[2]);
    real2 t2 = cadd(a[1], a[3]), t3 = csub(a[1], a[3]);
    real2 mt3 = mk2(t3.y, -t3.x);  // -i * t3
    a[0] = cadd(t0, t2);
    a[2] = csub(t0, t2);
    a[1] = cadd(t1, mt3);
    a[3] = csub(t1, mt3);
  } else if (R == 3) {
    const real s3 = 0.86602540378443864676;  // sin(2pi/3)
    real2 s = cadd(a[1], a[2]), d = csub(a[1], a[2]);
    real2 b0 = cadd(a[0], s);
    real2 m = mk2(a[0].x - real(0.5) * s.x, a[0].y - real(0.5) * s.y);
    real2 r = mk2(s3 * d.y, -s3 * d.x);  // -i sin(2pi/3) d
    a[0] = b0;
    a[1] = cadd(m, r);
    a[2] = csub(m, r);
  } else if (R == 5) {
    const real c1 = 0.30901699437494742410, c2 = -0.80901699437494742410;
    const real s1 = 0.95105651629515357212, s2 = 0.58778525229247312917;
    real2 t1 = cadd(a[1], a[4]), t2 = cadd(a[2], a[3]);
    real2 t3 = csub(a[1], a[4]), t4 = csub(a[2], a[3]);
    real2 b0 = cadd(a[0], cadd(t1, t2));
    real2 m1 = mk2(a[0].x + c1 * t1.x + c2 * t2.x, a[0].y + c1 * t1.y + c2 * t2.y);
    real2 m2 = mk2(a[0].x + c2 * t1.x + c1 * t2.x, a[0].y + c2 * t1.y + c1 * t2.y);
    // -i (s1 t3 + s2 t4) and -i (s2 t3 - s1 t4)
    real2 n1 = mk2(s1 * t3.y + s2 * t4.y, -(s1 * t3.x + s2 * t4.x));
    real2 n2 = mk2(s2 * t3.y - s1 * t4.y, -(s2 * t3.x - s1 * t4.x));
    a[0] = b0;
    a[1] = cadd(m1, n1);
    a[4] = csub(m1, n1);
    a[2] = cadd(m2, n2);
    a[3] = csub(m2, n2);
  }
}

template <int R>
__device__ __forceinline__ void stage(const real2* __restrict__ src, real2* __restrict__ dst, int n, int len,
                                      int nrows, int stride_row, const real2* __restrict__ tw) {
  const int m = len / R, s = n / len;
  const int nb = m * s;  // butterflies per row
  for (int e = threadIdx.x; e < nb * nrows; e += blockDim.x) {
    int row = e / nb, b = e - row * nb;
    int p = b / s, q = b - p * s;
    const real2* S = src + (size_t)row * stride_row;
    real2* D = dst + (size_t)row * stride_row;
    real2 a[R];
#pragma unroll
    for (int r = 0; r < R; ++r) a[r] = S[q + s * (p + r * m)];
    small_dft<R>(a);
    D[q + s * (R * p)] = a[0];
#pragma unroll
    for (int t = 1; t < R; ++t) D[q + s * (R * p + t)] = cmul(a[t], tw[p * R + t]);
  }
}

// Forward complex FFT of nrows rows held in buf0 (stride_row); buf1 is the
// ping-pong workspace.  Returns the buffer holding the result.
__device__ real2* fft_rows(real2* buf0, real2* buf1, int nrows, int stride_row, const FftPlan& pl,
                             const real2* __restrict__ twbase) {
  real2* src = buf0;
  real2* dst = buf1;
  int len = pl.n;
  for (int st = 0; st < pl.nst; ++st) {
    const real2* tw = twbase + pl.tw_off[st];
    switch (pl.radix[st]) {
      case 4: stage<4>(src, dst, pl.n, len, nrows, stride_row, tw); break;
      case 2: stage<2>(src, dst, pl.n, len, nrows, stride_row, tw); break;
      case 3: stage<3>(src, dst, pl.n, len, nrows, stride_row, tw); break;
      case 5: stage<5>(src, dst, pl.n, len, nrows, stride_row, tw); break;
    }
    __syncthreads();
    len /= pl.radix[st];
    real2* t = src;
    src = dst;
    dst = t;
  }
  return src;
}

// ---- forward y pass: phys -> mid ------------------------------------------------
// CTA: one z level, TXF consecutive x columns (TXF/2 complex rows of length Ny).
__global__ void __launch_bounds__(FFT_THREADS) k_fwd_y(Geom g, int TXF, FftPlan pl, const real2* __restrict__ tw,
                                                       const real* __restrict__ phys, real* __restrict__ mid) {
  extern __shared__ real2 sm[];
  const int Ny = g.Ny, Nx = g.Nx;
  const int nr = TXF / 2;
  real2* b0 = sm;
  real2* b1 = sm + (size_t)nr * Ny;
  const int x0 = blockIdx.x * TXF, k = blockIdx.y;
  const real* P = phys + (size_t)k * Ny * Nx;
  for (int e = threadIdx.x; e < Ny * TXF; e += blockDim.x) {
    int j = e / TXF, x = e - j * TXF;
    real v = P[(size_t)j * Nx + x0 + x];
    real* c = (real*)&b0[(x >> 1) * Ny + j];
    c[x & 1] = v;
  }
  __syncthreads();
  real2* res = fft_rows(b0, b1, nr, Ny, pl, tw);
  real* M = mid + (size_t)k * g.sy * Nx;
  const int half = Ny / 2 + 1;
  for (int e = threadIdx.x; e < half * TXF; e += blockDim.x) {
    int a = e / TXF, x = e - a * TXF;
    int r = x >> 1;
    real2 z1 = res[r * Ny + a];
    real2 z2 = res[r * Ny + (a == 0 ? 0 : Ny - a)];
    real re, im;
    if ((x & 1) == 0) {  // A = (Z_a + conj Z_{N-a}) / 2
      re = real(0.5) * (z1.x + z2.x);
      im = real(0.5) * (z1.y - z2.y);
    } else {             // B = (Z_a - conj Z_{N-a}) / (2i)
      re = real(0.5) * (z1.y + z2.y);
      im = real(-0.5) * (z1.x - z2.x);
    }
    M[(size_t)(2 * a) * Nx + x0 + x] = re;
    M[(size_t)(2 * a + 1) * Nx + x0 + x] = im;
  }
}

// ---- forward x pass: mid -> spec ------------------------------------------------
// CTA: RP pairs of consecutive rows (row = (k, j') flattened), rows of length Nx.
__global__ void __launch_bounds__(FFT_THREADS) k_fwd_x(Geom g, int RP, int64_t nrows_total, FftPlan pl,
                                                       const real2* __restrict__ tw, const real* __restrict__ mid,
                                                       real* __restrict__ spec) {
  extern __shared__ real2 sm[];
  const int Nx = g.Nx;
  real2* b0 = sm;
  real2* b1 = sm + (size_t)RP * Nx;
  const int64_t row0 = (int64_t)blockIdx.x * RP * 2;
  for (int e = threadIdx.x; e < RP * 2 * Nx; e += blockDim.x) {
    int rr = e / Nx, i = e - rr * Nx;
    int64_t row = row0 + rr;
    real v = row < nrows_total ? mid[(size_t)row * Nx + i] : real(0);
    real* c = (real*)&b0[(rr >> 1) * Nx + i];
    c[rr & 1] = v;
  }
  __syncthreads();
  real2* res = fft_rows(b0, b1, RP, Nx, pl, tw);
  const int half = Nx / 2 + 1;
  for (int e = threadIdx.x; e < RP * 2 * half; e += blockDim.x) {
    int rr = e / half, b = e - rr * half;
    int64_t row = row0 + rr;
    if (row >= nrows_total) continue;
    int r = rr >> 1;
    real2 z1 = res[r * Nx + b];
    real2 z2 = res[r * Nx + (b == 0 ? 0 : Nx - b)];
    real re, im;
    if ((rr & 1) == 0) {
      re = real(0.5) * (z1.x + z2.x);
      im = real(0.5) * (z1.y - z2.y);
    } else {
      re = real(0.5) * (z1.y + z2.y);
      im = real(-0.5) * (z1.x - z2.x);
    }
    spec[(size_t)row * g.sx + 2 * b] = re;
    spec[(size_t)row * g.sx + 2 * b + 1] = im;
  }
}

// Build Z_k = A_k + i B_k over the full circle from two half spectra, applying
// ffte_c2r's conjugate-symmetric fill (ffte_mod.F90:108-113): for k > N/2,
// A_k = conj(A_{N-k}); the imaginary parts of modes 0 and N/2 never reach the
// real output, so they are dropped.  Stored conjugated (FFTE computes the
// inverse as conj(FFT(conj(Z)))/N, vzfft1d.f:41-46, 63-68).
__device__ __forceinline__ real2 c2r_pack(real2 A, real2 B, int k, int n) {
  // A, B are the half-spectrum values at min(k, n-k); mirrored if k > n/2
  if (k == 0 || 2 * k == n) {
    A.y = real(0);
    B.y = real(0);
  }
  real2 z;
  if (2 * k <= n) {
    z = mk2(A.x - B.y, A.y + B.x);  // A + iB
  } else {
    // conj(A) + i conj(B) = (A.x + B.y) + i(-A.y + B.x)
    z = mk2(A.x + B.y, -A.y + B.x);
  }
  return mk2(z.x, -z.y);  // conj for the forward-transform inverse
}

// The spectral values A (row ra) and B (row ra + 1) of x mode km as the
// inverse x pass reads them, with the input operator applied.  ra is even and
// Ny + 2 is even, so row ra holds the even y' index jp (the real part of a y
// mode) and row ra + 1 the odd one of the same level lev; each value is the
// element pair (2 km, 2 km + 1) of its row.  The operators repeat the
// arithmetic of diffx, diffy and the filter (spectral_impl.cuh: dx_of, dy_of,
// k_filter) and the velocity spectra of vort2vel.F90:251-320 (e - diffy(c),
// diffx(c) - e, diffy(a) - diffx(b); the mean flow in mode (0, 0) of u and v).
// own: this thread reads mode km unmirrored, so it stores the filtered
// velocity spectrum of SPEC_VEL.
__device__ __forceinline__ real2 ld2(const real* __restrict__ p, size_t i) { return *(const real2*)&p[i]; }
__device__ __forceinline__ void st2(real* __restrict__ p, size_t i, real2 v) { *(real2*)&p[i] = v; }

// The operator on the values of one spectral element pair of rows ra (xa)
// and ra + 1 (xb); ca, cb are their spectral columns, lev their level.  For
// SPEC_VEL x is e (u, v) or a (w) and y is c (u, v) or b (w).  The wavenumber
// tables are laid out like the spectra but kx depends on the x index alone and
// ky on the row alone, so kx is read from row 0 (x2 = 2 km, the pair's x
// index) and ky from column 0 of rows ca - x2 and cb - x2: the same values,
// one small L1-resident row or a per-thread constant instead of a second
// spectrum-sized read per element.
template <int OP>
__device__ __forceinline__ void spec_op(const SpecIn<real>& S, real2 xa, real2 xb, real2 ya, real2 yb, int ca, int cb,
                                        int x2, int lev, real2& A, real2& B) {
  auto kxp = [&](const real* t) { return ld2(t, x2); };
  auto kyp = [&](const real* t, int c) { const real v = t[c - x2]; return mk2(v, v); };
  if constexpr (OP == SPEC_VEL) {
    if (S.vmode == 0) {  // f = e - diffy(c), f(:,1,1) = ubar
      const real2 ta = kyp(S.ky, ca), tb = kyp(S.ky, cb);
      A = mk2(xa.x - (real(-1) * yb.x) * ta.x, xa.y - (real(-1) * yb.y) * ta.y);
      B = mk2(xb.x - ya.x * tb.x, xb.y - ya.y * tb.y);
      if (ca == 0) A.x = (real)S.zbar[lev];
    } else if (S.vmode == 1) {  // f = diffx(c) - e, f(:,1,1) = vbar
      const real2 ta = kxp(S.kx), tb = ta;
      A = mk2((real(-1) * ya.y) * ta.x - xa.x, ya.x * ta.y - xa.y);
      B = mk2((real(-1) * yb.y) * tb.x - xb.x, yb.x * tb.y - xb.y);
      if (ca == 0) A.x = (real)S.zbar[lev];
    } else {  // f = diffy(a) - diffx(b)
      const real2 ya2 = kyp(S.ky, ca), yb2 = kyp(S.ky, cb), xa2 = kxp(S.kx), xb2 = xa2;
      A = mk2((real(-1) * xb.x) * ya2.x - (real(-1) * ya.y) * xa2.x, (real(-1) * xb.y) * ya2.y - ya.x * xa2.y);
      B = mk2(xa.x * yb2.x - (real(-1) * yb.y) * xb2.x, xa.y * yb2.y - yb.x * xb2.y);
    }
  } else if constexpr (OP == SPEC_DX) {  // tab = kx
    const real2 ta = kxp(S.tab), tb = ta;
    A = mk2((real(-1) * xa.y) * ta.x, xa.x * ta.y);
    B = mk2((real(-1) * xb.y) * tb.x, xb.x * tb.y);
  } else if constexpr (OP == SPEC_DY) {  // tab = ky
    const real2 ta = kyp(S.tab, ca), tb = kyp(S.tab, cb);
    A = mk2((real(-1) * xb.x) * ta.x, (real(-1) * xb.y) * ta.y);
    B = mk2(xa.x * tb.x, xa.y * tb.y);
  } else if constexpr (OP == SPEC_FILT) {
    const real2 ta = ld2(S.tab, ca), tb = ld2(S.tab, cb);
    A = mk2(xa.x * ta.x, xa.y * ta.y);
    B = mk2(xb.x * tb.x, xb.y * tb.y);
  } else {
    A = xa;
    B = xb;
  }
}
// the filtered copy of a velocity spectrum pair (SPEC_VEL), at elements ea, eb
__device__ __forceinline__ void vel_store(const SpecIn<real>& S, size_t ea, size_t eb, int ca, int cb, real2 A,
                                          real2 B) {
  const real2 fa = ld2(S.filt, ca), fb = ld2(S.filt, cb);
  st2(S.fs, ea, mk2(A.x * fa.x, A.y * fa.y));
  st2(S.fs, eb, mk2(B.x * fb.x, B.y * fb.y));
}
// the operator's inputs of the element pair read from global memory
template <int OP>
__device__ __forceinline__ void spec_pair(const Geom& g, const real* __restrict__ spec, const SpecIn<real>& S,
                                          int64_t ra, int jp, int lev, int km, bool own, real2& A, real2& B) {
  const size_t ea = (size_t)ra * g.sx + 2 * km, eb = ea + g.sx;
  const int ca = jp * g.sx + 2 * km, cb = ca + g.sx;  // spectral columns of elements ea, eb
  if constexpr (OP == SPEC_VEL) {
    const real* x = S.vmode == 2 ? S.a : S.e;
    const real* y = S.vmode == 2 ? S.b : S.c;
    spec_op<OP>(S, ld2(x, ea), ld2(x, eb), ld2(y, ea), ld2(y, eb), ca, cb, 2 * km, lev, A, B);
    if (own) vel_store(S, ea, eb, ca, cb, A, B);
  } else {
    const real2 a = ld2(spec, ea), b = ld2(spec, eb);
    spec_op<OP>(S, a, b, a, b, ca, cb, 2 * km, lev, A, B);
  }
}
// the same with the operator chosen at run time (generic-length path)
__device__ __forceinline__ void spec_pair_rt(const Geom& g, const real* __restrict__ spec, const SpecIn<real>& S,
                                             int64_t ra, int jp, int lev, int km, bool own, real2& A, real2& B) {
  switch (S.op) {
    case SPEC_DX: spec_pair<SPEC_DX>(g, spec, S, ra, jp, lev, km, own, A, B); break;
    case SPEC_DY: spec_pair<SPEC_DY>(g, spec, S, ra, jp, lev, km, own, A, B); break;
    case SPEC_FILT: spec_pair<SPEC_FILT>(g, spec, S, ra, jp, lev, km, own, A, B); break;
    case SPEC_VEL: spec_pair<SPEC_VEL>(g, spec, S, ra, jp, lev, km, own, A, B); break;
    default: spec_pair<SPEC_PLAIN>(g, spec, S, ra, jp, lev, km, own, A, B); break;
  }
}

// the output operator of an inverse transform at physical element i, v the
// transformed value: the pointwise updates of vorticity_tendency.F90 in its
// order of operations (dp :169-171, :180-181, :191-193; dq :213-214,
// :224-225, :235-237; dr :250-264, with v = dw/dy)
template <int OP>
__device__ __forceinline__ real phys_op(const PhysOut<real>& E, size_t i, real v, real& o2) {
  const real o = E.o[i];
  if constexpr (OP == PHYS_ADD_MUL) return o + E.in[0][i] * v;
  if constexpr (OP == PHYS_ADD_MUL_SUM) return o + E.in[0][i] * (E.in[1][i] + v);
  if constexpr (OP == PHYS_NEG_ADD_MUL) return -o + E.in[0][i] * v;
  if constexpr (OP == PHYS_DQ_DR) {
    const real r = E.in[0][i], p = E.in[1][i];
    real w = p * E.in[3][i];
    w = w + E.in[2][i] * v;
    w = w + r * (-E.in[4][i]);
    w = w + r * (-E.in[5][i]);
    o2 = w;
    return o + r * (-p + v);
  }
  return o;
}
// two consecutive elements i, i + 1 (i even, rows of even length)
template <int OP>
__device__ __forceinline__ void phys_out2(const PhysOut<real>& E, real* __restrict__ phys, size_t i, real2 v) {
  if (OP == PHYS_STORE || E.store) st2(phys, i, v);
  if constexpr (OP != PHYS_STORE) {
    real w0 = real(0), w1 = real(0);
    const real o0 = phys_op<OP>(E, i, v.x, w0);
    const real o1 = phys_op<OP>(E, i + 1, v.y, w1);
    st2(E.o, i, mk2(o0, o1));
    if constexpr (OP == PHYS_DQ_DR) st2(E.o2, i, mk2(w0, w1));
  }
}
// one element, the operator chosen at run time (generic-length path)
__device__ __forceinline__ void phys_out_rt(const PhysOut<real>& E, real* __restrict__ phys, size_t i, real v) {
  if (E.op == PHYS_STORE || E.store) phys[i] = v;
  real w = real(0);
  switch (E.op) {
    case PHYS_ADD_MUL: E.o[i] = phys_op<PHYS_ADD_MUL>(E, i, v, w); break;
    case PHYS_ADD_MUL_SUM: E.o[i] = phys_op<PHYS_ADD_MUL_SUM>(E, i, v, w); break;
    case PHYS_NEG_ADD_MUL: E.o[i] = phys_op<PHYS_NEG_ADD_MUL>(E, i, v, w); break;
    case PHYS_DQ_DR:
      E.o[i] = phys_op<PHYS_DQ_DR>(E, i, v, w);
      E.o2[i] = w;
      break;
    default: break;
  }
}

// ---- inverse x pass: spec -> mid ------------------------------------------------
__global__ void __launch_bounds__(FFT_THREADS) k_inv_x(Geom g, int RP, int64_t nrows_total, FftPlan pl,
                                                       const real2* __restrict__ tw, const real* __restrict__ spec,
                                                       real* __restrict__ mid, SpecIn<real> S) {
  extern __shared__ real2 sm[];
  const int Nx = g.Nx;
  real2* b0 = sm;
  real2* b1 = sm + (size_t)RP * Nx;
  const int64_t row0 = (int64_t)blockIdx.x * RP * 2;
  for (int e = threadIdx.x; e < RP * Nx; e += blockDim.x) {
    int r = e / Nx, k = e - r * Nx;
    int km = (2 * k <= Nx) ? k : Nx - k;
    int64_t ra = row0 + 2 * r;
    real2 A = mk2(real(0), real(0)), B = mk2(real(0), real(0));
    if (ra < nrows_total) {
      const int lev = (int)(ra / g.sy);
      spec_pair_rt(g, spec, S, ra, (int)(ra - (int64_t)lev * g.sy), lev, km, 2 * k <= Nx, A, B);
    }
    b0[r * Nx + k] = c2r_pack(A, B, k, Nx);
  }
  __syncthreads();
  real2* res = fft_rows(b0, b1, RP, Nx, pl, tw);
  const real dn = real(1) / (real)Nx;
  for (int e = threadIdx.x; e < RP * 2 * Nx; e += blockDim.x) {
    int rr = e / Nx, i = e - rr * Nx;
    int64_t row = row0 + rr;
    if (row >= nrows_total) continue;
    real2 z = res[(rr >> 1) * Nx + i];
    // conj(z) * dn: real part -> row A, imaginary part -> row B
    mid[(size_t)row * Nx + i] = (rr & 1) == 0 ? z.x * dn : -z.y * dn;
  }
}

// ---- inverse y pass: mid -> phys ------------------------------------------------
__global__ void __launch_bounds__(FFT_THREADS) k_inv_y(Geom g, int TXF, FftPlan pl, const real2* __restrict__ tw,
                                                       const real* __restrict__ mid, real* __restrict__ phys,
                                                       PhysOut<real> E) {
  extern __shared__ real2 sm[];
  const int Ny = g.Ny, Nx = g.Nx;
  const int nr = TXF / 2;
  real2* b0 = sm;
  real2* b1 = sm + (size_t)nr * Ny;
  const int x0 = blockIdx.x * TXF, k = blockIdx.y;
  const real* M = mid + (size_t)k * g.sy * Nx;
  // stage the half spectra (Ny/2+1 modes x TXF columns) into b1 first
  const int half = Ny / 2 + 1;
  for (int e = threadIdx.x; e < half * TXF; e += blockDim.x) {
    int a = e / TXF, x = e - a * TXF;
    b1[x * half + a] = mk2(M[(size_t)(2 * a) * Nx + x0 + x], M[(size_t)(2 * a + 1) * Nx + x0 + x]);
  }
  __syncthreads();
  for (int e = threadIdx.x; e < nr * Ny; e += blockDim.x) {
    int r = e / Ny, kk = e - r * Ny;
    int km = (2 * kk <= Ny) ? kk : Ny - kk;
    real2 A = b1[(2 * r) * half + km], B = b1[(2 * r + 1) * half + km];
    b0[r * Ny + kk] = c2r_pack(A, B, kk, Ny);
  }
  __syncthreads();
  real2* res = fft_rows(b0, b1, nr, Ny, pl, tw);
  const real dn = real(1) / (real)Ny;
  const size_t p0 = (size_t)k * Ny * Nx;
  for (int e = threadIdx.x; e < Ny * TXF; e += blockDim.x) {
    int j = e / TXF, x = e - j * TXF;
    real2 z = res[(x >> 1) * Ny + j];
    phys_out_rt(E, phys, p0 + (size_t)j * Nx + x0 + x, (x & 1) == 0 ? z.x * dn : -z.y * dn);
  }
}

// ---- four-step register FFT for n = n1 * n2, n1, n2 in {4, 8, 16} --------------------
// x[n2 + N2 n1] -> X[k1 + N1 k2]:  n1-point DFTs over n1 (one thread per n2),
// twiddle W_n^(n2 k1), transpose through shared memory, n2-point DFTs over n2
// (one thread per k1).  The small DFTs run in registers; loads and stores touch
// global memory once each.

// W_16^m = exp(-2 pi i m / 16), m known at compile time after unrolling
__device__ __forceinline__ real2 w16(int m) {
  constexpr real C1 = 0.92387953251128675613;  // cos(pi/8)
  constexpr real C2 = 0.70710678118654752440;  // cos(pi/4)
  constexpr real C3 = 0.38268343236508977173;  // cos(3pi/8)
  switch (m & 15) {
    case 0: return mk2(1.0, 0.0);
    case 1: return mk2(C1, -C3);
    case 2: return mk2(C2, -C2);
    case 3: return mk2(C3, -C1);
    case 4: return mk2(0.0, -1.0);
    case 5: return mk2(-C3, -C1);
    case 6: return mk2(-C2, -C2);
    case 7: return mk2(-C1, -C3);
    case 8: return mk2(-1.0, 0.0);
    case 9: return mk2(-C1, C3);
    case 10: return mk2(-C2, C2);
    case 11: return mk2(-C3, C1);
    case 12: return mk2(0.0, 1.0);
    case 13: return mk2(C3, C1);
    case 14: return mk2(C2, C2);
    default: return mk2(C1, C3);
  }
}

// forward DFT of size R in registers, natural order in and out
template <int R>
__device__ __forceinline__ void dft(real2* a) {
  if constexpr (R <= 5) {
    small_dft<R>(a);
  } else {
    constexpr int M1 = 4, M2 = R / 4;  // R = 8: 4 x 2, R = 16: 4 x 4
    real2 y[R];
#pragma unroll
    for (int n2 = 0; n2 < M2; ++n2) {
      real2 b[M1];
#pragma unroll
      for (int n1 = 0; n1 < M1; ++n1) b[n1] = a[M2 * n1 + n2];
      small_dft<M1>(b);
#pragma unroll
      for (int k1 = 0; k1 < M1; ++k1) y[k1 * M2 + n2] = (n2 * k1 == 0) ? b[k1] : cmul(b[k1], w16(n2 * k1 * (16 / R)));
    }
#pragma unroll
    for (int k1 = 0; k1 < M1; ++k1) {
      real2 c[M2];
#pragma unroll
      for (int n2 = 0; n2 < M2; ++n2) c[n2] = y[k1 * M2 + n2];
      small_dft<M2>(c);
#pragma unroll
      for (int k2 = 0; k2 < M2; ++k2) a[k1 + M1 * k2] = c[k2];
    }
  }
}


// step 1 of one row: a[n1] = x[n2 + N2 n1] on entry; Y row [k1][n2] (padded)
template <int N1, int N2>
__device__ __forceinline__ void fs_step1(real2* a, int n2, real2* Yrow, const real2* __restrict__ tw4) {
  dft<N1>(a);
#pragma unroll
  for (int k1 = 0; k1 < N1; ++k1) Yrow[k1 * (N2 + 1) + n2] = (k1 == 0 || n2 == 0) ? a[k1] : cmul(a[k1], tw4[n2 * N1 + k1]);
}
// step 3 of one row: a[k2] = X[k1 + N1 k2] on return
template <int N1, int N2>
__device__ __forceinline__ void fs_step3(real2* a, int k1, const real2* Yrow) {
#pragma unroll
  for (int n2 = 0; n2 < N2; ++n2) a[n2] = Yrow[k1 * (N2 + 1) + n2];
  dft<N2>(a);
}

// forward x pass (mid -> spec): RP complex rows (pairs of real rows) per CTA
template <int N1, int N2>
__global__ void __launch_bounds__(FS_THREADS) k4_fwd_x(Geom g, int64_t nrows_total, const real2* __restrict__ tw4,
                                                       const real* __restrict__ mid, real* __restrict__ spec) {
  constexpr int N = N1 * N2, RP = FS_THREADS / (N1 > N2 ? N1 : N2), YS = N1 * (N2 + 1);
  __shared__ real2 Y[RP * YS];
  real2* X = Y;  // [RP][N], reuses Y after step 3 has read it
  const int t = threadIdx.x;
  const int64_t row0 = (int64_t)blockIdx.x * RP * 2;
  if (t < RP * N2) {
    const int r = t / N2, n2 = t % N2;
    const int64_t ra = row0 + 2 * r, rb = ra + 1;
    real2 a[N1];
#pragma unroll
    for (int n1 = 0; n1 < N1; ++n1) {
      const int i = n2 + N2 * n1;
      a[n1] = mk2(ra < nrows_total ? mid[(size_t)ra * N + i] : real(0),
                           rb < nrows_total ? mid[(size_t)rb * N + i] : real(0));
    }
    fs_step1<N1, N2>(a, n2, Y + r * YS, tw4);
  }
  __syncthreads();
  {  // every thread reaches the barrier; RP * N1 <= FS_THREADS
    const bool act = t < RP * N1;
    const int r = t / N1, k1 = t % N1;
    real2 a[N2];
    if (act) fs_step3<N1, N2>(a, k1, Y + r * YS);
    __syncthreads();
#pragma unroll
    for (int k2 = 0; k2 < N2; ++k2)
      if (act) X[r * N + k1 + N1 * k2] = a[k2];
  }
  __syncthreads();
  // separate the two real rows: A = (Z_b + conj Z_{N-b}) / 2, B = (Z_b - conj Z_{N-b}) / (2i)
  constexpr int HALF = N / 2 + 1;
  for (int e = t; e < RP * 2 * HALF; e += FS_THREADS) {
    const int rr = e / HALF, b = e - rr * HALF;
    const int64_t row = row0 + rr;
    if (row >= nrows_total) continue;
    const int r = rr >> 1;
    const real2 z1 = X[r * N + b];
    const real2 z2 = X[r * N + (b == 0 ? 0 : N - b)];
    real re, im;
    if ((rr & 1) == 0) {
      re = real(0.5) * (z1.x + z2.x);
      im = real(0.5) * (z1.y - z2.y);
    } else {
      re = real(0.5) * (z1.y + z2.y);
      im = real(-0.5) * (z1.x - z2.x);
    }
    spec[(size_t)row * g.sx + 2 * b] = re;
    spec[(size_t)row * g.sx + 2 * b + 1] = im;
  }
}

// inverse x pass (spec -> mid).  The modes are read straight from HBM into
// registers (the mirrored half from L1), the input operator applied on the
// way.  Both transform passes are bound by L1 / shared-memory throughput, not
// HBM, so no extra staging pass through shared memory is made.
template <int N1, int N2, int OP>
__global__ void __launch_bounds__(FS_THREADS) k4_inv_x(Geom g, int64_t nrows_total, const real2* __restrict__ tw4,
                                                       const real* __restrict__ spec, real* __restrict__ mid,
                                                       SpecIn<real> S) {
  constexpr int N = N1 * N2, RP = FS_THREADS / (N1 > N2 ? N1 : N2), YS = N1 * (N2 + 1);
  __shared__ real2 Y[RP * YS];
  const int t = threadIdx.x;
  const int64_t row0 = (int64_t)blockIdx.x * RP * 2;
  if (t < RP * N2) {
    const int r = t / N2, n2 = t % N2;
    const int64_t ra = row0 + 2 * r;
    const bool valid = ra < nrows_total;  // then so is ra + 1: the row count is even
    const int lev = (int)(ra / g.sy), jp = (int)(ra - (int64_t)lev * g.sy);
    real2 a[N1];
#pragma unroll
    for (int n1 = 0; n1 < N1; ++n1) {
      const int k = n2 + N2 * n1;
      const int km = (2 * k <= N) ? k : N - k;
      real2 A = mk2(real(0), real(0)), B = mk2(real(0), real(0));
      if (valid) spec_pair<OP>(g, spec, S, ra, jp, lev, km, 2 * k <= N, A, B);
      a[n1] = c2r_pack(A, B, k, N);
    }
    fs_step1<N1, N2>(a, n2, Y + r * YS, tw4);
  }
  __syncthreads();
  const real dn = real(1) / (real)N;
  if (t < RP * N1) {
    const int r = t / N1, k1 = t % N1;
    real2 a[N2];
    fs_step3<N1, N2>(a, k1, Y + r * YS);
    const int64_t ra = row0 + 2 * r, rb = ra + 1;
#pragma unroll
    for (int k2 = 0; k2 < N2; ++k2) {
      const int i = k1 + N1 * k2;  // conj(z) * dn: real part -> row A, imaginary part -> row B
      if (ra < nrows_total) mid[(size_t)ra * N + i] = a[k2].x * dn;
      if (rb < nrows_total) mid[(size_t)rb * N + i] = -a[k2].y * dn;
    }
  }
}

// forward y pass (phys -> mid): one z level, 16 consecutive x columns
// (8 complex columns) per CTA; thread order puts consecutive x on consecutive threads
template <int N1, int N2>
__global__ void __launch_bounds__(FS_THREADS) k4_fwd_y(Geom g, const real2* __restrict__ tw4,
                                                       const real* __restrict__ phys, real* __restrict__ mid) {
  // rows of Y and X are padded so the 8 column pairs of a warp access fall in
  // distinct shared-memory banks
  constexpr int N = N1 * N2, RP = 8, YS = N1 * (N2 + 1) + 1, XS = N + 1;
  __shared__ real2 Y[RP * YS];
  real2* X = Y;  // [RP][XS], reuses Y after step 3 has read it
  const int t = threadIdx.x, Nx = g.Nx;
  const int x0 = blockIdx.x * 2 * RP, k = blockIdx.y;
  const real* P = phys + (size_t)k * N * Nx;
  if (t < RP * N2) {
    const int r = t % RP, n2 = t / RP;
    real2 a[N1];
#pragma unroll
    for (int n1 = 0; n1 < N1; ++n1) {
      const int j = n2 + N2 * n1;
      a[n1] = *(const real2*)&P[(size_t)j * Nx + x0 + 2 * r];  // columns x0+2r (re), x0+2r+1 (im)
    }
    fs_step1<N1, N2>(a, n2, Y + r * YS, tw4);
  }
  __syncthreads();
  {  // every thread reaches the barrier; RP * N1 <= FS_THREADS
    const bool act = t < RP * N1;
    const int r = t % RP, k1 = t / RP;
    real2 a[N2];
    if (act) fs_step3<N1, N2>(a, k1, Y + r * YS);
    __syncthreads();
#pragma unroll
    for (int k2 = 0; k2 < N2; ++k2)
      if (act) X[r * XS + k1 + N1 * k2] = a[k2];
  }
  __syncthreads();
  constexpr int HALF = N / 2 + 1;
  real* M = mid + (size_t)k * g.sy * Nx;
  for (int e = t; e < HALF * 2 * RP; e += FS_THREADS) {
    const int a = e / (2 * RP), x = e - a * (2 * RP);
    const int r = x >> 1;
    const real2 z1 = X[r * XS + a];
    const real2 z2 = X[r * XS + (a == 0 ? 0 : N - a)];
    real re, im;
    if ((x & 1) == 0) {
      re = real(0.5) * (z1.x + z2.x);
      im = real(0.5) * (z1.y - z2.y);
    } else {
      re = real(0.5) * (z1.y + z2.y);
      im = real(-0.5) * (z1.x - z2.x);
    }
    M[(size_t)(2 * a) * Nx + x0 + x] = re;
    M[(size_t)(2 * a + 1) * Nx + x0 + x] = im;
  }
}

// inverse y pass (mid -> phys)
template <int N1, int N2, int OP>
__global__ void __launch_bounds__(FS_THREADS) k4_inv_y(Geom g, const real2* __restrict__ tw4,
                                                       const real* __restrict__ mid, real* __restrict__ phys,
                                                       PhysOut<real> E) {
  // rows of Y and X are padded so the 8 column pairs of a warp access fall in
  // distinct shared-memory banks
  constexpr int N = N1 * N2, RP = 8, YS = N1 * (N2 + 1) + 1;
  __shared__ real2 Y[RP * YS];
  const int t = threadIdx.x, Nx = g.Nx;
  const int x0 = blockIdx.x * 2 * RP, k = blockIdx.y;
  const real* M = mid + (size_t)k * g.sy * Nx;
  if (t < RP * N2) {
    const int r = t % RP, n2 = t / RP;
    real2 a[N1];
#pragma unroll
    for (int n1 = 0; n1 < N1; ++n1) {
      const int kk = n2 + N2 * n1;
      const int km = (2 * kk <= N) ? kk : N - kk;
      const real2 re = *(const real2*)&M[(size_t)(2 * km) * Nx + x0 + 2 * r];      // (A.re, B.re)
      const real2 im = *(const real2*)&M[(size_t)(2 * km + 1) * Nx + x0 + 2 * r];  // (A.im, B.im)
      a[n1] = c2r_pack(mk2(re.x, im.x), mk2(re.y, im.y), kk, N);
    }
    fs_step1<N1, N2>(a, n2, Y + r * YS, tw4);
  }
  __syncthreads();
  const real dn = real(1) / (real)N;
  if (t < RP * N1) {
    const int r = t % RP, k1 = t / RP;
    real2 a[N2];
    fs_step3<N1, N2>(a, k1, Y + r * YS);
    const size_t p0 = (size_t)k * N * Nx + x0 + 2 * r;
#pragma unroll
    for (int k2 = 0; k2 < N2; ++k2)
      phys_out2<OP>(E, phys, p0 + (size_t)(k1 + N1 * k2) * Nx, mk2(a[k2].x * dn, -a[k2].y * dn));
  }
}

// launchers by split; return false if the split has no instantiation
#define PMPIC_FS_CASES(CALL) \
  if (n1 == 4 && n2 == 4) { CALL(4, 4); return true; } \
  if (n1 == 8 && n2 == 4) { CALL(8, 4); return true; } \
  if (n1 == 8 && n2 == 8) { CALL(8, 8); return true; } \
  if (n1 == 16 && n2 == 8) { CALL(16, 8); return true; } \
  if (n1 == 16 && n2 == 16) { CALL(16, 16); return true; } \
  return false;

bool fs_fwd_x(int n1, int n2, unsigned nb, cudaStream_t st, const Geom& g, int64_t nrows, const real2* tw4,
              const real* mid, real* spec) {
#define CALL(A, B) k4_fwd_x<A, B><<<nb, FS_THREADS, 0, st>>>(g, nrows, tw4, mid, spec)
  PMPIC_FS_CASES(CALL)
#undef CALL
}
template <int OP>
bool fs_inv_x_op(int n1, int n2, unsigned nb, cudaStream_t st, const Geom& g, int64_t nrows, const real2* tw4,
                 const real* spec, real* mid, const SpecIn<real>& S) {
#define CALL(A, B) k4_inv_x<A, B, OP><<<nb, FS_THREADS, 0, st>>>(g, nrows, tw4, spec, mid, S)
  PMPIC_FS_CASES(CALL)
#undef CALL
}
bool fs_inv_x(int n1, int n2, unsigned nb, cudaStream_t st, const Geom& g, int64_t nrows, const real2* tw4,
              const real* spec, real* mid, const SpecIn<real>& S) {
  switch (S.op) {
    case SPEC_DX: return fs_inv_x_op<SPEC_DX>(n1, n2, nb, st, g, nrows, tw4, spec, mid, S);
    case SPEC_DY: return fs_inv_x_op<SPEC_DY>(n1, n2, nb, st, g, nrows, tw4, spec, mid, S);
    case SPEC_FILT: return fs_inv_x_op<SPEC_FILT>(n1, n2, nb, st, g, nrows, tw4, spec, mid, S);
    case SPEC_VEL: return fs_inv_x_op<SPEC_VEL>(n1, n2, nb, st, g, nrows, tw4, spec, mid, S);
    default: return fs_inv_x_op<SPEC_PLAIN>(n1, n2, nb, st, g, nrows, tw4, spec, mid, S);
  }
}
bool fs_fwd_y(int n1, int n2, dim3 gr, cudaStream_t st, const Geom& g, const real2* tw4, const real* phys,
              real* mid) {
#define CALL(A, B) k4_fwd_y<A, B><<<gr, FS_THREADS, 0, st>>>(g, tw4, phys, mid)
  PMPIC_FS_CASES(CALL)
#undef CALL
}
template <int OP>
bool fs_inv_y_op(int n1, int n2, dim3 gr, cudaStream_t st, const Geom& g, const real2* tw4, const real* mid,
                 real* phys, const PhysOut<real>& E) {
#define CALL(A, B) k4_inv_y<A, B, OP><<<gr, FS_THREADS, 0, st>>>(g, tw4, mid, phys, E)
  PMPIC_FS_CASES(CALL)
#undef CALL
}
bool fs_inv_y(int n1, int n2, dim3 gr, cudaStream_t st, const Geom& g, const real2* tw4, const real* mid,
              real* phys, const PhysOut<real>& E) {
  switch (E.op) {
    case PHYS_ADD_MUL: return fs_inv_y_op<PHYS_ADD_MUL>(n1, n2, gr, st, g, tw4, mid, phys, E);
    case PHYS_ADD_MUL_SUM: return fs_inv_y_op<PHYS_ADD_MUL_SUM>(n1, n2, gr, st, g, tw4, mid, phys, E);
    case PHYS_NEG_ADD_MUL: return fs_inv_y_op<PHYS_NEG_ADD_MUL>(n1, n2, gr, st, g, tw4, mid, phys, E);
    case PHYS_DQ_DR: return fs_inv_y_op<PHYS_DQ_DR>(n1, n2, gr, st, g, tw4, mid, phys, E);
    default: return fs_inv_y_op<PHYS_STORE>(n1, n2, gr, st, g, tw4, mid, phys, E);
  }
}
#undef PMPIC_FS_CASES

int fft_forward_impl(pmpic_ctx* ctx, const real* phys, real* spec, real* mid, const real2* tw) {
  TimerScope ts(ctx, T_FFTF);
  const Geom& g = ctx->g;
  const FftPlan& px = ctx->plan_x;
  const FftPlan& py = ctx->plan_y;
  const real2* twy = tw + ctx->ftw_off_y;
  if (py.n1) {
    fs_fwd_y(py.n1, py.n2, dim3(g.Nx / 16, g.nzp), ctx->stream, g, twy + py.tw4_off, phys, mid);
  } else {
    int txf = pick_txf(g.Nx);
    size_t sm_y = sizeof(real2) * (size_t)(txf / 2) * g.Ny * 2;
    dim3 gy(g.Nx / txf, g.nzp);
    k_fwd_y<<<gy, FFT_THREADS, sm_y, ctx->stream>>>(g, txf, py, twy, phys, mid);
  }
  ++ctx->nlaunch;
  int64_t nrows = (int64_t)g.nzp * g.sy;
  if (px.n1) {
    const int rp = FS_THREADS / std::max(px.n1, px.n2);
    fs_fwd_x(px.n1, px.n2, (unsigned)((nrows + 2 * rp - 1) / (2 * rp)), ctx->stream, g, nrows, tw + px.tw4_off,
             mid, spec);
  } else {
    int rp = pick_rp(g.Nx);
    size_t sm_x = sizeof(real2) * (size_t)rp * g.Nx * 2;
    k_fwd_x<<<(unsigned)((nrows + 2 * rp - 1) / (2 * rp)), FFT_THREADS, sm_x, ctx->stream>>>(g, rp, nrows, px, tw,
                                                                                          mid, spec);
  }
  ++ctx->nlaunch;
  PMPIC_CUDA(cudaGetLastError());
  return 0;
}

int fft_backward_impl(pmpic_ctx* ctx, const real* spec, real* phys, real* mid, const real2* tw, const SpecIn<real>& S,
                      const PhysOut<real>& E) {
  TimerScope ts(ctx, T_FFTI);
  const Geom& g = ctx->g;
  const FftPlan& px = ctx->plan_x;
  const FftPlan& py = ctx->plan_y;
  int64_t nrows = (int64_t)g.nzp * g.sy;
  if (px.n1) {
    const int rp = FS_THREADS / std::max(px.n1, px.n2);
    fs_inv_x(px.n1, px.n2, (unsigned)((nrows + 2 * rp - 1) / (2 * rp)), ctx->stream, g, nrows, tw + px.tw4_off,
             spec, mid, S);
  } else {
    int rp = pick_rp(g.Nx);
    size_t sm_x = sizeof(real2) * (size_t)rp * g.Nx * 2;
    k_inv_x<<<(unsigned)((nrows + 2 * rp - 1) / (2 * rp)), FFT_THREADS, sm_x, ctx->stream>>>(g, rp, nrows, px, tw,
                                                                                          spec, mid, S);
  }
  ++ctx->nlaunch;
  const real2* twy = tw + ctx->ftw_off_y;
  if (py.n1) {
    fs_inv_y(py.n1, py.n2, dim3(g.Nx / 16, g.nzp), ctx->stream, g, twy + py.tw4_off, mid, phys, E);
  } else {
    int txf = pick_txf(g.Nx);
    size_t half = (size_t)g.Ny / 2 + 1;
    size_t sm_y = sizeof(real2) * std::max((size_t)(txf / 2) * g.Ny * 2, (size_t)(txf / 2) * g.Ny + txf * half);
    dim3 gy(g.Nx / txf, g.nzp);
    k_inv_y<<<gy, FFT_THREADS, sm_y, ctx->stream>>>(g, txf, py, twy, mid, phys, E);
  }
  ++ctx->nlaunch;
  PMPIC_CUDA(cudaGetLastError());
  return 0;
}


// shared-memory limits of the Stockham kernels (a property of each function on
// the current device)
cudaError_t fft_attributes() {
  cudaError_t e = cudaFuncSetAttribute(k_fwd_y, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
  if (e == cudaSuccess) e = cudaFuncSetAttribute(k_inv_y, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
  if (e == cudaSuccess) e = cudaFuncSetAttribute(k_fwd_x, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
  if (e == cudaSuccess) e = cudaFuncSetAttribute(k_inv_x, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
  return e;
}
