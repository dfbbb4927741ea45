// lbx_fused.cu — single-pass colour-gradient step (time_step_CG + streaming,
// kernels_fluid_CG.CUF:531-1141) for sm_100a, written for instruction
// economy: the collision of the two components shares the velocity factors
// of the equilibrium, opposite directions are processed as pairs (e_opp =
// -e_l, so every odd power of e.u / e.psi changes sign and every even power
// is shared), and all per-class products (omega rho_k w_l, the perturbation
// and recolouring coefficients) are formed once per cell.
//
// Schedule: a CTA of TX x TY threads owns the column [x0, x0+TX) x [y0, y0+TY)
// and marches it along z over one segment.  In iteration z it
//   1. pulls the populations of plane z+1 for its own cells and for the
//      one-cell ring around the column, and writes their phase field into a
//      rolling four-slot shared-memory window (only sums are formed, nothing
//      is kept in registers);
//   2. after one barrier, pulls the populations of plane z again (they are
//      L1/L2 resident from step 1 of the previous iteration), computes the
//      colour gradient from the window and collides, and stores the 38
//      post-collision populations of each cell with aligned, coalesced writes.
// The phase field never goes through global memory; the extra cost is the
// ring and the two boundary planes of each segment, read from L2.
#include "lbx_device.cuh"

namespace lbx {

template <typename C>
struct LeanConst {
  C w[3], b[3], a27[4];
  C sqrt2;
  C omega;           // uniform relaxation (tauR == tauB), else negative
  C inv_viscR, inv_viscB, inv_cssq;
  C sigma, beta;
  C rho0[2];         // shift densities of the stored populations (0 when unshifted)
  C s[2][3];         // shift of each weight class, w_cls * rho0
};

template <typename C>
LeanConst<C> make_lean(const Ctx& c) {
  LeanConst<C> K;
  LatticeT<C> L = make_lattice<C>();
  for (int i = 0; i < 3; ++i) { K.w[i] = L.w[i]; K.b[i] = L.b[i]; }
  for (int i = 0; i < 4; ++i) K.a27[i] = L.a27[i];
  K.sqrt2 = L.rec[2];
  const C HALF = C(0.5);
  C viscR = L.cssq * (C(c.p.tauR) - HALF), viscB = L.cssq * (C(c.p.tauB) - HALF);
  K.inv_viscR = C(1) / viscR;
  K.inv_viscB = C(1) / viscB;
  K.inv_cssq = L.inv_cssq;
  K.omega = (c.p.tauR == c.p.tauB) ? C(1) / (viscR / L.cssq + HALF) : C(-1);
  K.sigma = C(c.p.sigma);
  K.beta = C(c.p.beta);
  bool shifted = (c.storage == LBX_STORE_F16 || c.storage == LBX_STORE_BF16);
  K.rho0[0] = shifted ? C(c.p.rho0R) : C(0);
  K.rho0[1] = shifted ? C(c.p.rho0B) : C(0);
  for (int comp = 0; comp < 2; ++comp)
    for (int k = 0; k < 3; ++k) K.s[comp][k] = K.w[k] * K.rho0[comp];
  return K;
}

// raw stored value -> arithmetic type (no shift)
template <typename S> __device__ __forceinline__ float raw(S v);
template <> __device__ __forceinline__ float raw<float>(float v) { return v; }
template <> __device__ __forceinline__ float raw<__half>(__half v) { return __half2float(v); }
template <> __device__ __forceinline__ float raw<__nv_bfloat16>(__nv_bfloat16 v) { return __bfloat162float(v); }
__device__ __forceinline__ double raw_d(double v) { return v; }

template <typename S, typename C>
__device__ __forceinline__ C load_raw(const S* p) {
  if constexpr (std::is_same<S, double>::value) return __ldg(p);
  else return raw<S>(__ldg(p));
}
template <typename S, typename C>
__device__ __forceinline__ void store_raw(S* p, C v) {
  if constexpr (std::is_same<S, double>::value || std::is_same<S, float>::value) *p = v;
  else if constexpr (std::is_same<S, __half>::value) *p = __float2half_rn(v);
  else *p = __float2bfloat16_rn(v);
}

// 32-bit source offsets of the 19 pulls of a cell
struct PullIdx {
  int src[Q];
};

__device__ __forceinline__ void pull_idx(const Geom& g, int x, int y, int z, PullIdx& P) {
  int xm = (x == 0) ? g.nx - 1 : x - 1, xp = (x == g.nx - 1) ? 0 : x + 1;
  int ym = (y == 0) ? g.ny - 1 : y - 1, yp = (y == g.ny - 1) ? 0 : y + 1;
  int zm = (z == 0) ? g.nz - 1 : z - 1, zp = (z == g.nz - 1) ? 0 : z + 1;
  const int X[3] = {xm, x, xp};
  const int Y[3] = {ym * g.nx, y * g.nx, yp * g.nx};
  const int plane = g.nx * g.ny;
  const int Z[3] = {zm * plane, z * plane, zp * plane};
#pragma unroll
  for (int l = 0; l < Q; ++l) P.src[l] = X[1 - ex(l)] + Y[1 - ey(l)] + Z[1 - ez(l)];
}

// clamped densities (Sum g + rho0, init_rho*_CG) of the pulled cell
template <typename S, typename C>
__device__ __forceinline__ void pull_rho(const S* __restrict__ A, int64_t n, const PullIdx& P, const LeanConst<C>& K,
                                         C& rR, C& rB) {
  const S* aR = A;
  const S* aB = A + size_t(Q) * size_t(n);
  C sR = load_raw<S, C>(aR + P.src[0]);
  C sB = load_raw<S, C>(aB + P.src[0]);
#pragma unroll
  for (int l = 1; l < Q; ++l) {
    sR = sR + load_raw<S, C>(aR + size_t(l) * size_t(n) + P.src[l]);
    sB = sB + load_raw<S, C>(aB + size_t(l) * size_t(n) + P.src[l]);
  }
  rR = sR + K.rho0[0];
  rB = sB + K.rho0[1];
}

template <typename C>
__device__ __forceinline__ C clamp0(C v) { return v < C(0) ? C(0) : v; }

// One colour-gradient collision (time_step_CG, kernels_fluid_CG.CUF:689-846).
// gR/gB: stored-form populations (f - shift) on entry, post-collision stored
// form on exit.  rR/rB: clamped densities.
template <typename C>
__device__ __forceinline__ void collide_lean(const LeanConst<C>& K, C gR[Q], C gB[Q], C rR, C rB, C px, C py, C pz) {
  const C ONE = C(1), HALF = C(0.5);
  const C rs = rR + rB;
  C omega;
  if (K.omega >= C(0)) {
    omega = K.omega;
  } else {
    const C ph = (rR - rB) / rs;
    const C visc = ONE / (HALF * (ONE + ph) * K.inv_viscR + HALF * (ONE - ph) * K.inv_viscB);
    omega = ONE / (visc * K.inv_cssq + HALF);
  }
  const C omm = ONE - omega;
  const C inv = ONE / rs;
  // momentum of both components; the shifts cancel in every antisymmetric sum
  C S[Q];
#pragma unroll
  for (int l = 0; l < Q; ++l) S[l] = gR[l] + gB[l];
  const C u = inv * (S[1] - S[2] + S[7] - S[8] - S[9] + S[10] + S[11] - S[12] - S[13] + S[14]);
  const C v = inv * (S[3] - S[4] + S[7] - S[8] + S[9] - S[10] + S[15] - S[16] - S[17] + S[18]);
  const C w = inv * (S[5] - S[6] + S[11] - S[12] + S[13] - S[14] + S[15] - S[16] + S[17] - S[18]);
  const C c0 = ONE - C(1.5) * (u * u + v * v + w * w);
  // omega * rho_k * w_cls, and the shift of each class folded into the relaxation
  C KR[3], KB[3], sR[3], sB[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    KR[k] = omega * rR * K.w[k];
    KB[k] = omega * rB * K.w[k];
    sR[k] = K.s[0][k];
    sB[k] = K.s[1][k];
  }
  // BGK: f' = f (1 - omega) + omega rho w A,  f = g + s
  {
    const C a0 = c0;
    gR[0] = (gR[0] + sR[0]) * omm + KR[0] * a0;
    gB[0] = (gB[0] + sB[0]) * omm + KB[0] * a0;
  }
#pragma unroll
  for (int p = 1; p <= 9; ++p) {
    const int l = 2 * p - 1, o = 2 * p, k = wclass(l);
    const C eu = edot(l, u, v, w);
    const C P = c0 + C(4.5) * eu * eu;
    const C Qv = C(3) * eu;
    const C Ap = P + Qv, Am = P - Qv;
    gR[l] = (gR[l] + sR[k]) * omm + KR[k] * Ap;
    gR[o] = (gR[o] + sR[k]) * omm + KR[k] * Am;
    gB[l] = (gB[l] + sB[k]) * omm + KB[k] * Ap;
    gB[o] = (gB[o] + sB[k]) * omm + KB[k] * Am;
  }
  const C psq = px * px + py * py + pz * pz;
  const C kR = rR * inv, kB = rB * inv;
  if (psq > C(1.e-20)) {
    const C pn = sqrt(psq);
    const C ipn = ONE / pn;
    const C acoeff = C(9) / C(4) * omega * K.sigma;
    const C coef = K.beta * rR * rB * inv * ipn;  // beta rR rB / (rs |psi|)
    C K1[3], K0[3], K3[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      K1[k] = acoeff * K.w[k] * ipn;  // acoeff |psi| w / |psi|^2
      K0[k] = acoeff * pn * K.b[k];
    }
    K3[0] = C(0);
    K3[1] = coef * K.w[1];
    K3[2] = coef * K.w[2] / K.sqrt2;
    {
      const C fd = gR[0] + gB[0] - K0[0];
      gR[0] = fd * kR - sR[0];
      gB[0] = fd * kB - sB[0];
    }
#pragma unroll
    for (int p = 1; p <= 9; ++p) {
      const int l = 2 * p - 1, o = 2 * p, k = wclass(l);
      const C ed = edot(l, px, py, pz);
      const C pert = K1[k] * (ed * ed) - K0[k];
      const C T = K3[k] * ed;
      const C fdp = gR[l] + gB[l] + pert;
      const C fdm = gR[o] + gB[o] + pert;
      gR[l] = fdp * kR + (T - sR[k]);
      gB[l] = fdp * kB - (T + sB[k]);
      gR[o] = fdm * kR - (T + sR[k]);
      gB[o] = fdm * kB + (T - sB[k]);
    }
  } else {
    gR[0] -= sR[0];
    gB[0] -= sB[0];
#pragma unroll
    for (int p = 1; p <= 9; ++p) {
      const int l = 2 * p - 1, o = 2 * p, k = wclass(l);
      gR[l] -= sR[k]; gR[o] -= sR[k];
      gB[l] -= sB[k]; gB[o] -= sB[k];
    }
  }
}

template <int TX, int TY>
struct Ring {
  static constexpr int RX = TX + 2, RY = TY + 2, CELLS = RX * RY, N = 2 * RX + 2 * TY, NT = TX * TY;
};

__device__ __forceinline__ int wrap0(int v, int n) {
  v %= n;
  return v < 0 ? v + n : v;
}

// Particle data of a step (flags of this and of the previous step, the side
// densities written by the fill and wetting kernels, written back here for
// every fluid cell for the bounce-back of the same step and the drain of the
// next).
template <typename C>
struct LeanPart {
  const int8_t* __restrict__ fold;
  const int8_t* __restrict__ fnew;
  C* rhoR;
  C* rhoB;
};

template <typename S, int TX, int TY, int MINB, bool PART>
__global__ void __launch_bounds__(TX* TY, MINB)
    k_cg_lean(const S* __restrict__ A, S* __restrict__ B, Geom g, LeanConst<typename Store<S>::C> K, int zlen,
              unsigned long long* err, int64_t step, LeanPart<typename Store<S>::C> PT) {
  using C = typename Store<S>::C;
  using R = Ring<TX, TY>;
  __shared__ C sphi[4][R::CELLS];
  const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * TX + tx;
  const int x0 = blockIdx.x * TX, y0 = blockIdx.y * TY, z0 = blockIdx.z * zlen;
  const int zend = min(z0 + zlen, g.nz);
  const bool active = (x0 + tx < g.nx) && (y0 + ty < g.ny);
  const int x = wrap0(x0 + tx, g.nx), y = wrap0(y0 + ty, g.ny);
  const int own = (ty + 1) * R::RX + (tx + 1);
  // ring cell of this thread (threads 0 .. N-1)
  int rx = 0, ry = 0;
  const bool ringer = tid < R::N;
  if (tid < R::RX) { rx = tid; ry = 0; }
  else if (tid < 2 * R::RX) { rx = tid - R::RX; ry = R::RY - 1; }
  else if (tid < 2 * R::RX + TY) { rx = 0; ry = 1 + tid - 2 * R::RX; }
  else { rx = R::RX - 1; ry = 1 + tid - 2 * R::RX - TY; }
  const int rxg = wrap0(x0 + rx - 1, g.nx), ryg = wrap0(y0 + ry - 1, g.ny);
  const int rslot = ry * R::RX + rx;

  // clamped densities of cell (cx, cy, zz): pulled (fluid in both steps),
  // from the side arrays (new fluid, or the virtual density of a surface
  // cell), zero for every other solid cell (init_rho*_CG's MINDENS)
  auto densities = [&](int cx, int cy, int zz, bool check, C& rR, C& rB) {
    const int cell = cx + g.nx * (cy + g.ny * zz);
    if constexpr (PART) {
      const int8_t fn = PT.fnew[cell];
      if (fn != LBX_FLUID_FLUID) {
        if (fn == LBX_FLUID_SPHERELIST) { rR = PT.rhoR[cell]; rB = PT.rhoB[cell]; }
        else { rR = C(0); rB = C(0); }
        return false;
      }
      if (PT.fold[cell] != LBX_FLUID_FLUID) {
        rR = PT.rhoR[cell];
        rB = PT.rhoB[cell];
        return false;
      }
    }
    PullIdx P;
    pull_idx(g, cx, cy, zz, P);
    pull_rho<S, C>(A, g.n, P, K, rR, rB);
    if (check && (rR < C(-10) || rR > C(10) || rB < C(-10) || rB > C(10)))
      raise_error(err, LBX_DEV_RHO_RANGE, step, cell);
    rR = clamp0(rR);
    rB = clamp0(rB);
    return true;
  };

  // phase field of plane z (own cell and ring cell) into slot
  auto phase_plane = [&](int z, int slot, C& rRo, C& rBo) {
    const int zz = wrap0(z, g.nz);
    const bool owned = active && z >= z0 && z < zend;
    C rR, rB;
    const bool pulled = densities(x, y, zz, owned, rR, rB);
    if constexpr (PART) {
      if (owned && pulled) {  // the densities of init_rho*_CG for the particle kernels
        const int cell = x + g.nx * (y + g.ny * zz);
        PT.rhoR[cell] = rR;
        PT.rhoB[cell] = rB;
      }
    }
    (void)pulled;
    rRo = rR;
    rBo = rB;
    sphi[slot][own] = (rR - rB) / (rR + rB);
    if (ringer) {
      C qR, qB;
      densities(rxg, ryg, zz, false, qR, qB);
      sphi[slot][rslot] = (qR - qB) / (qR + qB);
    }
  };

  C rRn, rBn, rRc, rBc;
  phase_plane(z0 - 1, (z0 + 3) & 3, rRc, rBc);
  phase_plane(z0, z0 & 3, rRn, rBn);
  for (int z = z0; z < zend; ++z) {
    rRc = rRn;
    rBc = rBn;
    phase_plane(z + 1, (z + 1) & 3, rRn, rBn);
    __syncthreads();
    if (active) {
      const int cell = x + g.nx * (y + g.ny * z);
      PullIdx P;
      pull_idx(g, x, y, z, P);
      C gR[Q], gB[Q];
      const S* aB = A + size_t(Q) * size_t(g.n);
      S* bR = B + cell;
      S* bB = B + size_t(Q) * size_t(g.n) + cell;
      bool collide = true;
      if constexpr (PART) {
        const int8_t fn = PT.fnew[cell], fo = PT.fold[cell];
        collide = fn == LBX_FLUID_FLUID;
        if (collide && fo != LBX_FLUID_FLUID) {
          // make_fluid already wrote the new node's populations (stored form) into B
#pragma unroll
          for (int l = 0; l < Q; ++l) {
            gR[l] = load_raw<S, C>(bR + size_t(l) * size_t(g.n));
            gB[l] = load_raw<S, C>(bB + size_t(l) * size_t(g.n));
          }
        } else if (!collide) {
          // solid cell: streamed populations only; a spheredead source (previous
          // step) leaves the destination's stale value, which is B's entry
#pragma unroll
          for (int l = 0; l < Q; ++l) {
            const bool dead = l > 0 && PT.fold[P.src[l]] == LBX_FLUID_SPHEREDEAD;
            gR[l] = dead ? load_raw<S, C>(bR + size_t(l) * size_t(g.n))
                         : load_raw<S, C>(A + size_t(l) * size_t(g.n) + P.src[l]);
            gB[l] = dead ? load_raw<S, C>(bB + size_t(l) * size_t(g.n))
                         : load_raw<S, C>(aB + size_t(l) * size_t(g.n) + P.src[l]);
          }
        } else {
#pragma unroll
          for (int l = 0; l < Q; ++l) {
            gR[l] = load_raw<S, C>(A + size_t(l) * size_t(g.n) + P.src[l]);
            gB[l] = load_raw<S, C>(aB + size_t(l) * size_t(g.n) + P.src[l]);
          }
        }
      } else {
#pragma unroll
        for (int l = 0; l < Q; ++l) {
          gR[l] = load_raw<S, C>(A + size_t(l) * size_t(g.n) + P.src[l]);
          gB[l] = load_raw<S, C>(aB + size_t(l) * size_t(g.n) + P.src[l]);
        }
      }
      if (collide) {
        const C* pm = sphi[(z + 3) & 3];
        const C* p0 = sphi[z & 3];
        const C* pp = sphi[(z + 1) & 3];
        C px = 0, py = 0, pz = 0;
#pragma unroll
        for (int l = 1; l < Q27; ++l) {
          const int dx = ex27(l), dy = ey27(l), dz = ez27(l);
          const C* pl = dz < 0 ? pm : (dz > 0 ? pp : p0);
          const C ps = pl[own + dy * R::RX + dx];
          const C a = K.a27[wclass27(l)];
          if (dx) px = px + (dx > 0 ? a : -a) * ps;
          if (dy) py = py + (dy > 0 ? a : -a) * ps;
          if (dz) pz = pz + (dz > 0 ? a : -a) * ps;
        }
        collide_lean(K, gR, gB, rRc, rBc, px, py, pz);
      }
#pragma unroll
      for (int l = 0; l < Q; ++l) {
        store_raw<S, C>(bR + size_t(l) * size_t(g.n), gR[l]);
        store_raw<S, C>(bB + size_t(l) * size_t(g.n), gB[l]);
      }
    }
    // slot (z+3)&3 read above is rewritten in iteration z+2; the barrier of
    // iteration z+1 orders that write after these reads
  }
}

// ---------------------------------------------------------------------------
static int lean_zlen(const Ctx& c, int tx, int ty, int per_sm) {
  long cols = long((c.nx + tx - 1) / tx) * long((c.ny + ty - 1) / ty);
  long target = 148L * per_sm * 2;
  long segs = (target + cols - 1) / cols;
  if (segs < 1) segs = 1;
  if (segs > c.nz) segs = c.nz;
  return int((c.nz + segs - 1) / segs);
}

template <typename S, int TX, int TY, int MINB, bool PART>
static void launch_lean(Ctx& c, int zlen_override, LeanPart<typename Store<S>::C> pt) {
  using C = typename Store<S>::C;
  int zlen = zlen_override > 0 ? zlen_override : lean_zlen(c, TX, TY, MINB);
  dim3 block(TX, TY, 1);
  dim3 grid((c.nx + TX - 1) / TX, (c.ny + TY - 1) / TY, (c.nz + zlen - 1) / zlen);
  k_cg_lean<S, TX, TY, MINB, PART><<<grid, block, 0, c.stream>>>(
      (const S*)c.pops[c.cur], (S*)c.pops[1 - c.cur], geom(c), make_lean<C>(c), zlen, c.d_err, c.step + 1, pt);
}

void kt_begin(Ctx& c);
void kt_end(Ctx& c);

// shape: 0 = 32x8 (two CTAs per SM), 1 = 32x16 (one CTA per SM)
int fluid_lean(Ctx& c) {
  int rc = by_storage(c, [&](auto* tag) {
    using S = std::remove_pointer_t<decltype(tag)>;
    using C = typename Store<S>::C;
    LeanPart<C> none{nullptr, nullptr, nullptr, nullptr};
    kt_begin(c);
    if constexpr (std::is_same<S, double>::value) {
      launch_lean<S, 32, 8, 1, false>(c, c.lean_zlen, none);
    } else {
      if (c.lean_shape == 1) launch_lean<S, 32, 16, 1, false>(c, c.lean_zlen, none);
      else launch_lean<S, 32, 8, 2, false>(c, c.lean_zlen, none);
    }
    kt_end(c);
    return launch_status();
  });
  if (!rc) c.cur = 1 - c.cur;
  return rc;
}

// the same step with particle flags (fo: flags of the previous step, fn: of this one)
int fluid_lean_particles(Ctx& c, int fo, int fn) {
  int rc = by_storage(c, [&](auto* tag) {
    using S = std::remove_pointer_t<decltype(tag)>;
    using C = typename Store<S>::C;
    LeanPart<C> pt{c.flags[fo], c.flags[fn], (C*)c.rho[0], (C*)c.rho[1]};
    kt_begin(c);
    if constexpr (std::is_same<S, double>::value) launch_lean<S, 32, 8, 1, true>(c, c.lean_zlen, pt);
    else launch_lean<S, 32, 8, 2, true>(c, c.lean_zlen, pt);
    kt_end(c);
    return launch_status();
  });
  return rc;  // the particle step swaps the buffers after its bounce-back
}

}  // namespace lbx
