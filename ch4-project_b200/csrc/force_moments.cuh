// Global corrections of build_forcing (included by lb_kernels.cuh inside namespace ch4).
//
// LB_FLUID_FORCING_NOZEROMODE (src/forcing.c:1123-1152) subtracts the volume mean
// of the force field; LB_FLUID_FORCING_CONSTANT_POWER (src/forcing.c:1154-1190) then
// scales component a by Amp_a / fac, fac = <F . u> over the volume, with u the
// velocity field of the last hydro_fields.  Both need the whole field before any
// cell can use its force, so one reduction pass runs ahead of the step kernel:
// per cell the raw force F^n (from t^n = m(g^n), s^n = m(h^n) and the current
// tables), and with CONSTANT_POWER also u^n = mv/rho + dt/2 F^{n-1}.  Nine sums
// (F, F*u, u per component) run in double-double over a fixed cell -> block
// assignment and a fixed tree, so the result is deterministic; the final kernel
// forms fm = {f0, coeff} in FP64.  The reference sums sequentially, so with these
// flags the FP64 path agrees with it to rounding, not bit for bit.

template <typename S, typename A, bool THERM, bool SCAL>
__global__ void __launch_bounds__(FM_BLOCK)
    force_sums_kernel(const StepParams<A> P, const A* hit_cur, int with_prev, double* partial) {
  constexpr bool EXACT = sizeof(A) == 8;
  __shared__ double sh_hi[FM_BLOCK], sh_lo[FM_BLOCK];
  const long long per_block = (P.N + gridDim.x - 1) / gridDim.x;
  const long long c0 = (long long)blockIdx.x * per_block;
  const long long c1 = c0 + per_block < P.N ? c0 + per_block : P.N;
  const bool cpower = (P.feat & K_CPOWER) != 0;
  DD acc[FM_SUMS];
  for (int q = 0; q < FM_SUMS; q++) acc[q] = {0.0, 0.0};
  for (long long idx = c0 + threadIdx.x; idx < c1; idx += FM_BLOCK) {
    const int x = (int)(idx % P.NX);
    const int y = (int)((idx / P.NX) % P.NY);
    const int z = (int)(idx / ((long long)P.NX * P.NY));
    A tt = A(0), ss = A(0);
    if constexpr (THERM) {
      A g[Q];
      load_set<S, A, 1>(P, idx, g);
      tt = mom0(g);
    }
    if constexpr (SCAL) {
      A h[Q];
      load_set<S, A, 2>(P, idx, h);
      ss = mom0(h);
    }
    A fx, fy, fz;
    cell_force(P, x, y, z, idx, tt, ss, hit_cur, (const A*)nullptr, (const A*)nullptr, fx, fy, fz);
    acc[0] = dd_add(acc[0], (double)fx);
    acc[1] = dd_add(acc[1], (double)fy);
    acc[2] = dd_add(acc[2], (double)fz);
    if (cpower) {
      A f[Q];
      load_set<S, A, 0>(P, idx, f);
      const A rho = mom0(f);
      A px = A(0), py = A(0), pz = A(0);
      if (with_prev) {
        const A tp = THERM ? P.tprev[idx] : A(0);
        const A sp = SCAL ? P.sprev[idx] : A(0);
        cell_force(P, x, y, z, idx, tp, sp, P.hit_prev, (P.feat & K_TWOWAY) ? P.dprev : nullptr, P.fm_prev, px, py,
                   pz);
      }
      A ux, uy, uz;
      if constexpr (EXACT) {
        ux = momx(f) / rho + P.hdt * px;
        uy = momy(f) / rho + P.hdt * py;
        uz = momz(f) / rho + P.hdt * pz;
      } else {
        const A ir = A(1) / rho;
        ux = momx(f) * ir + P.hdt * px;
        uy = momy(f) * ir + P.hdt * py;
        uz = momz(f) * ir + P.hdt * pz;
      }
      acc[3] = dd_add(acc[3], (double)fx * (double)ux);
      acc[4] = dd_add(acc[4], (double)fy * (double)uy);
      acc[5] = dd_add(acc[5], (double)fz * (double)uz);
      acc[6] = dd_add(acc[6], (double)ux);
      acc[7] = dd_add(acc[7], (double)uy);
      acc[8] = dd_add(acc[8], (double)uz);
    }
  }
  for (int q = 0; q < FM_SUMS; q++) {
    sh_hi[threadIdx.x] = acc[q].hi;
    sh_lo[threadIdx.x] = acc[q].lo;
    __syncthreads();
    for (int w = FM_BLOCK / 2; w > 0; w >>= 1) {
      if ((int)threadIdx.x < w) {
        DD a = {sh_hi[threadIdx.x], sh_lo[threadIdx.x]};
        DD b = {sh_hi[threadIdx.x + w], sh_lo[threadIdx.x + w]};
        a = dd_add(a, b);
        sh_hi[threadIdx.x] = a.hi;
        sh_lo[threadIdx.x] = a.lo;
      }
      __syncthreads();
    }
    if (threadIdx.x == 0) {
      partial[((long long)blockIdx.x * FM_SUMS + q) * 2] = sh_hi[0];
      partial[((long long)blockIdx.x * FM_SUMS + q) * 2 + 1] = sh_lo[0];
    }
    __syncthreads();
  }
}

// fm = {f0x, f0y, f0z, coeffx, coeffy, coeffz} from the block partials (one thread)
template <typename A>
__global__ void force_final_kernel(const double* partial, int nblocks, int nozero, int cpower, double norm, double amp_x,
                                   double amp_y, double amp_z, A* fm) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  double sum[FM_SUMS];
  for (int q = 0; q < FM_SUMS; q++) {
    DD a = {0.0, 0.0};
    for (int b = 0; b < nblocks; b++)
      a = dd_add(a, DD{partial[((long long)b * FM_SUMS + q) * 2], partial[((long long)b * FM_SUMS + q) * 2 + 1]});
    sum[q] = a.hi + a.lo;
  }
  double f0[3] = {0.0, 0.0, 0.0}, coeff[3] = {1.0, 1.0, 1.0};
  if (nozero)
    for (int a = 0; a < 3; a++) f0[a] = sum[a] * norm;
  if (cpower) {
    // <(F - f0) . u> = sum F_a u_a - f0_a sum u_a, per component
    const double fac = ((sum[3] - f0[0] * sum[6]) + (sum[4] - f0[1] * sum[7]) + (sum[5] - f0[2] * sum[8])) * norm;
    if (fac != 0.0) {
      coeff[0] = amp_x / fac;
      coeff[1] = amp_y / fac;
      coeff[2] = amp_z / fac;
    }
  }
  for (int a = 0; a < 3; a++) {
    fm[a] = (A)f0[a];
    fm[3 + a] = (A)coeff[a];
  }
}
