// Ray ceilings: per daytime hour, an upper bound at every pixel q of the
// heights that the rest of a sun ray passing through q can still present,
// discounted by the ray's rise.  The shadow sweep uses it to stop walking a
// ray as soon as no later sample can change any of its outputs.
//
// The sweep of pixel p visits q_j = p + o_j (j = 0 .. K-1, o_j the ray table)
// and at step j compares the heights h in {dsm, canopy top, trunk} at q_j
// against the pixel through h - dz_j and h - dz_{j-1}.  Let H = max(dsm,
// vegdem, vegdem2).  If a value C(q_k) satisfies, for every pixel p whose ray
// visits q_k at step k and every later step j >= k,
//        H(q_j) - dz_{j-1}  <=  C(q_k) - dz_{k-1}                        (*)
// then C(q_k) - dz_{k-1} < dsm_p means no later sample reaches above the
// pixel (its shadow height, vegetation flags and, when also <= topmax, the
// canopy top seen by a wall are final).
//
// Construction (all bounds exact, no trigonometry):
//  * frame: the major axis is the one whose offset equals +-j at every step
//    (checked over the whole table); X runs along it in the ray direction and
//    Y along the other axis, oriented so the last offset is >= 0.  Then
//    X(q_j) = X(q_k) + (j - k) and Y(q_j) = Y(p) + m_j with m_j the minor
//    offset.
//  * shear: with v = M / D, M = m_{K-1}, D = K - 1, R(X) = floor(X M / D) in
//    integers and the sheared line N = Y - R(X).  Along one ray
//    N(q_j) - N(q_k) = (e_j - e_k) - (R(X_j) - R(X_k) - (j-k) v) with
//    e_i = m_i - i v, so |N(q_j) - N(q_k)| < spread(e) + 1, i.e. <= W with
//    W = floor(spread) + 1 (spread measured exactly as D * e_i in integers;
//    about 1 for the rounded digital rays, so W = 2).
//  * discount: delta = the smallest increment dz_i - dz_{i-1} of the table
//    (exact in float64 by Sterbenz), rounded down to float32, so
//    dz_{j-1} - dz_{k-1} >= (j - k) delta for j >= k >= 1.
//  * along each sheared line, G(X) = max(Hd(X), G(X+1) - delta) with
//    Hd(X, N) = max over |d| <= W of H(X, N + d + R(X)) and the subtraction
//    rounded up, so G(X, N) >= H(X', N') - (X' - X) delta for X' >= X and
//    |N' - N| <= W: C(q) = G(X(q), N(q)) satisfies (*) for k >= 1.
//
// The dilation runs along the raster's minor axis only, so it is done once
// per day (ceiling_dilate_kernel): H dilated by +-1 and +-2 along the columns
// (row-major planes, for rays whose major axis is the rows) and along the rows
// (stored transposed, for rays whose major axis is the columns).  Either way
// the scan reads plane[a * nb + b] with a the oriented major index and b the
// oriented minor index, so a warp's 32 lanes (consecutive Y) read 32
// consecutive floats.
//
// Window maxima: with the ceiling the scan also writes, per pixel,
// M(X, N) = max over X' in [X, X + kCeilSkip) of Hd(X', N) (no discount).  A
// ray through q_k at step k >= 1 meets q_{k..k+kCeilSkip-1} within +-W lines,
// so H(q_j) - dz_{j-1} <= M(q_k) - dz_{k-1} for those steps: when that is
// <= dsm_p none of their compares is above the pixel and a walk (not of a
// wall pixel) may skip them.  The planes hold (C, M) as float2 per pixel.
//
// Scan layout: a block owns 32 consecutive sheared lines (one per lane) and
// splits the major axis into 16 segments (one per warp; 512 threads, so two
// blocks fit per SM).  Phase 1 scans each
// segment backwards from -inf; phase 2 carries the later segments' maxima in
// and rescans, writing the plane.
#pragma once
#include "common.cuh"

namespace solweig {

constexpr int kCeilLanes = 32;     // sheared lines per block
constexpr int kCeilWarps = 16;     // major-axis segments per block
constexpr int kCeilMaxBand = 3;    // largest dilation W handled
constexpr int kCeilMinSteps = 5;   // the sweep consults the plane from step 4 on

// Upper bound (float32) of max(dsm, vegdem, vegdem2) at pixel p.
template <bool G32>
__device__ __forceinline__ float ceiling_height(const SolweigScene& S, long long p) {
    if (G32) {
        const float4 v = __ldg(reinterpret_cast<const float4*>(S.geo32) + p);
        return fmaxf(v.x, fmaxf(v.y, v.z));
    }
    const double m = fmax(__ldg(&S.dsm[p]), fmax(__ldg(&S.vegdem[p]), __ldg(&S.vegdem2[p])));
    return __double2float_ru(m);
}

struct CeilingFrame {
    int ok;            // 0: the table fits no frame; the plane is +inf
    int rows_major;    // major axis = rows (else columns)
    int s_major, s_minor;
    int nx, nb;        // extents along X (major) and Y (minor)
    int m, d;          // slope v = m / d of the shear
    int band;          // dilation W
    int lines;         // sheared lines: nb + R(nx - 1)
    float delta;       // per-step discount
};

// Frame of one hour's ray, derived by the whole block from the table.
__device__ inline CeilingFrame ceiling_frame(const SolweigScene& S, const int2* __restrict__ ray,
                                      const double* __restrict__ dz, int K) {
    __shared__ long long s_emin, s_emax;
    __shared__ unsigned s_dmin;
    const int tid = threadIdx.y * blockDim.x + threadIdx.x, nt = blockDim.x * blockDim.y;
    const int2 last = ray[K - 1];
    const int sr = last.x < 0 ? -1 : 1, sc = last.y < 0 ? -1 : 1;
    int rows_ok = 1, cols_ok = 1;
    for (int i = tid; i < K; i += nt) {
        const int2 o = __ldg(&ray[i]);
        rows_ok &= (o.x == sr * i);
        cols_ok &= (o.y == sc * i);
    }
    rows_ok = __syncthreads_and(rows_ok);
    cols_ok = __syncthreads_and(cols_ok);
    CeilingFrame f{};
    f.rows_major = rows_ok;
    f.ok = rows_ok || cols_ok;
    if (!f.ok) return f;
    f.s_major = rows_ok ? sr : sc;
    f.s_minor = rows_ok ? sc : sr;
    f.nx = rows_ok ? S.rows : S.cols;
    f.nb = rows_ok ? S.cols : S.rows;
    f.d = K - 1;
    f.m = f.s_minor * (rows_ok ? last.y : last.x);  // >= 0
    if (tid == 0) {
        s_emin = LLONG_MAX;
        s_emax = LLONG_MIN;
        s_dmin = 0x7f800000u;  // +inf
    }
    __syncthreads();
    long long emin = LLONG_MAX, emax = LLONG_MIN;
    float dmin = __int_as_float(0x7f800000);
    int inc_ok = 1;
    for (int i = tid; i < K; i += nt) {
        const int2 o = __ldg(&ray[i]);
        const long long mi = (long long)f.s_minor * (rows_ok ? o.y : o.x);
        const long long e = mi * f.d - (long long)i * f.m;  // D * e_i
        emin = min(emin, e);
        emax = max(emax, e);
        if (i >= 1) {
            const double inc = __ldg(&dz[i]) - __ldg(&dz[i - 1]);  // exact (Sterbenz)
            inc_ok &= (inc >= 0.0);                                 // false for NaN too
            if (inc >= 0.0) dmin = fminf(dmin, __double2float_rd(inc));
        }
    }
    atomicMin(&s_emin, emin);
    atomicMax(&s_emax, emax);
    atomicMin(&s_dmin, __float_as_uint(dmin));  // non-negative floats order as integers
    inc_ok = __syncthreads_and(inc_ok);
    const long long spread = s_emax - s_emin;  // D * spread(e)
    f.band = (int)(spread / f.d) + 1;
    f.delta = __uint_as_float(s_dmin);
    // (nx - 1) * m must fit the 32-bit shear cursor
    if (!inc_ok || f.m > f.d || f.band > kCeilMaxBand || (long long)(f.nx - 1) * f.m > INT_MAX) {
        f.ok = 0;
        return f;
    }
    f.lines = f.nb + (f.nx - 1) * f.m / f.d;
    return f;
}

__device__ __forceinline__ long long ceiling_pixel(const CeilingFrame& f, int cols, int x, int y) {
    const int a = f.s_major > 0 ? x : f.nx - 1 - x;
    const int b = f.s_minor > 0 ? y : f.nb - 1 - y;
    return f.rows_major ? (long long)a * cols + b : (long long)b * cols + a;
}

// R(X) = floor(X m / d) while X steps down by one: quotient and remainder
// carried in 32-bit integers (X m <= rows * cols), no division per step.
struct ShearCursor {
    int rx, rem;
    __device__ __forceinline__ ShearCursor(int x, int m, int d) {
        const int num = x * m;
        rx = num / d;
        rem = num - rx * d;
    }
    __device__ __forceinline__ void step_down(int m, int d) {  // m <= d
        rem -= m;
        if (rem < 0) {
            rem += d;
            --rx;
        }
    }
};

constexpr int kCeilBatch = 8;  // samples fetched ahead of the dependent max chain

// H dilated by +-W along the minor axis around Y = y at major index a:
// plane[a * nb + b].  A line whose centre lies up to W outside the raster
// still sees its in-raster neighbours: the edge pixel's window covers them.
__device__ __forceinline__ float ceiling_sample(const float* __restrict__ plane, const CeilingFrame& f, int a, int y) {
    if (y < -f.band || y >= f.nb + f.band) return __int_as_float(0xff800000);
    const int yc = min(max(y, 0), f.nb - 1);
    const int b = f.s_minor > 0 ? yc : f.nb - 1 - yc;
    return __ldg(&plane[(long long)a * f.nb + b]);
}

// One backward scan of [x0, x1) from g over the lane's sheared line; with OUT,
// writes every pixel of the line: (ceiling, window maximum).  A batch of loads
// is issued before the dependent chain consumes it.  win[i] holds Hd at
// x + 1 + i (the samples of the window after x), preloaded at the segment end.
template <bool OUT>
__device__ __forceinline__ float ceiling_run(const float* __restrict__ plane, const CeilingFrame& f, int cols,
                                             int line, int x0, int x1, float g, float2* __restrict__ out) {
    const float ninf = __int_as_float(0xff800000);
    float win[kCeilSkip - 1];
#pragma unroll
    for (int i = 0; i < kCeilSkip - 1; ++i) {
        win[i] = ninf;
        if (OUT && x1 + i < f.nx) {
            const int xx = x1 + i;
            const int a = f.s_major > 0 ? xx : f.nx - 1 - xx;
            win[i] = ceiling_sample(plane, f, a, line + (int)(((long long)xx * f.m) / f.d));
        }
    }
    auto emit = [&](int x, int y, float v) {
        float m = v;
#pragma unroll
        for (int i = 0; i < kCeilSkip - 1; ++i) m = fmaxf(m, win[i]);
#pragma unroll
        for (int i = kCeilSkip - 2; i > 0; --i) win[i] = win[i - 1];
        win[0] = v;
        if (OUT && y >= 0 && y < f.nb) out[ceiling_pixel(f, cols, x, y)] = make_float2(g, m);
    };
    ShearCursor cur(max(x1 - 1, 0), f.m, f.d);
    int x = x1 - 1;
    for (; x - (kCeilBatch - 1) >= x0; x -= kCeilBatch) {
        float v[kCeilBatch];
        int y[kCeilBatch];
#pragma unroll
        for (int u = 0; u < kCeilBatch; ++u) {
            y[u] = line + cur.rx;
            const int a = f.s_major > 0 ? x - u : f.nx - 1 - (x - u);
            v[u] = ceiling_sample(plane, f, a, y[u]);
            cur.step_down(f.m, f.d);
        }
#pragma unroll
        for (int u = 0; u < kCeilBatch; ++u) {
            g = fmaxf(v[u], __fsub_ru(g, f.delta));
            if (OUT) emit(x - u, y[u], v[u]);
        }
    }
    for (; x >= x0; --x) {
        const int yy = line + cur.rx;
        const int a = f.s_major > 0 ? x : f.nx - 1 - x;
        const float v = ceiling_sample(plane, f, a, yy);
        g = fmaxf(v, __fsub_ru(g, f.delta));
        if (OUT) emit(x, yy, v);
        cur.step_down(f.m, f.d);
    }
    return g;
}

// Both phases for one block of 32 sheared lines (see the file comment).
__device__ __forceinline__ void ceiling_scan(const float* __restrict__ plane, const CeilingFrame& f, int cols,
                                             int line0, float (*s_seg)[kCeilLanes], float2* __restrict__ out) {
    const int seg = (f.nx + kCeilWarps - 1) / kCeilWarps;
    const int w = threadIdx.y;
    const int x0 = min(f.nx, w * seg), x1 = min(f.nx, x0 + seg);
    const int line = line0 + threadIdx.x;
    const float ninf = __int_as_float(0xff800000);
    // phase 1: segment maxima from -inf
    s_seg[w][threadIdx.x] = ceiling_run<false>(plane, f, cols, line, x0, x1, ninf, nullptr);
    __syncthreads();
    // phase 2: carry of the later segments, then the rescan that writes
    float carry = ninf;
    for (int s = kCeilWarps - 1; s > w; --s) {
        const int s0 = min(f.nx, s * seg), s1 = min(f.nx, s0 + seg);
        carry = fmaxf(s_seg[s][threadIdx.x], __fsub_ru(carry, __fmul_rd((float)(s1 - s0), f.delta)));
    }
    ceiling_run<true>(plane, f, cols, line, x0, x1, carry, out);
}

// The four dilated planes of H (see the file comment), each rows x cols floats:
//   dil[0], dil[1]: +-1, +-2 along the columns, row-major [r][c];
//   dil[2], dil[3]: +-1, +-2 along the rows, transposed [c][r].
// block (32, 8) over a 32 x 32 tile, H staged with a 2-pixel halo.
constexpr int kDilTile = 32, kDilHalo = 2, kDilPitch = kDilTile + 2 * kDilHalo + 1;

template <bool G32>
__global__ void __launch_bounds__(256) ceiling_dilate_kernel(SolweigScene S, float* __restrict__ dil) {
    __shared__ float tile[kDilTile + 2 * kDilHalo][kDilPitch];
    const int r0 = blockIdx.y * kDilTile, c0 = blockIdx.x * kDilTile;
    const int tid = threadIdx.y * 32 + threadIdx.x;
    const float ninf = __int_as_float(0xff800000);
    constexpr int side = kDilTile + 2 * kDilHalo;
    for (int i = tid; i < side * side; i += 256) {
        const int tr = i / side, tc = i - tr * side;
        const int r = r0 - kDilHalo + tr, c = c0 - kDilHalo + tc;
        tile[tr][tc] = (r >= 0 && r < S.rows && c >= 0 && c < S.cols)
                           ? ceiling_height<G32>(S, (long long)r * S.cols + c) : ninf;
    }
    __syncthreads();
    const long long n = (long long)S.rows * S.cols;
    // along the columns: thread x = column (row-major writes coalesced)
    for (int k = threadIdx.y; k < kDilTile; k += 8) {
        const int r = r0 + k, c = c0 + threadIdx.x;
        if (r >= S.rows || c >= S.cols) continue;
        const float* t = &tile[k + kDilHalo][threadIdx.x + kDilHalo];
        const float d1 = fmaxf(t[0], fmaxf(t[-1], t[1]));
        const float d2 = fmaxf(d1, fmaxf(t[-2], t[2]));
        dil[(long long)r * S.cols + c] = d1;
        dil[n + (long long)r * S.cols + c] = d2;
    }
    // along the rows: thread x = row (transposed writes coalesced)
    for (int k = threadIdx.y; k < kDilTile; k += 8) {
        const int r = r0 + threadIdx.x, c = c0 + k;
        if (r >= S.rows || c >= S.cols) continue;
        const int tr = threadIdx.x + kDilHalo, tc = k + kDilHalo;
        const float d1 = fmaxf(tile[tr][tc], fmaxf(tile[tr - 1][tc], tile[tr + 1][tc]));
        const float d2 = fmaxf(d1, fmaxf(tile[tr - 2][tc], tile[tr + 2][tc]));
        dil[2 * n + (long long)c * S.rows + r] = d1;
        dil[3 * n + (long long)c * S.rows + r] = d2;
    }
}

// The ceiling plane of one ray table (K steps) for the raster of S, by one
// block of (32, kCeilWarps) threads owning 32 sheared lines (blockIdx.x); the whole
// block returns together.  Tables the frame does not fit give a +inf plane.
__device__ __forceinline__ void ray_ceiling_block(const SolweigScene& S, const int2* __restrict__ ray,
                                                  const double* __restrict__ dz, int K,
                                                  const float* __restrict__ dil, float2* __restrict__ out,
                                                  float (*s_seg)[kCeilLanes]) {
    if (K < kCeilMinSteps) return;
    const long long n = (long long)S.rows * S.cols;
    const CeilingFrame f = ceiling_frame(S, ray, dz, K);
    const int tid = threadIdx.y * kCeilLanes + threadIdx.x;
    if (!f.ok || f.band > 2) {
        for (long long p = (long long)blockIdx.x * blockDim.x * blockDim.y + tid; p < n;
             p += (long long)gridDim.x * blockDim.x * blockDim.y)
            out[p] = make_float2(__int_as_float(0x7f800000), __int_as_float(0x7f800000));
        return;
    }
    const int line_first = blockIdx.x * kCeilLanes;
    if (line_first >= f.lines) return;
    // lane l owns sheared line N = line_first + l - R(nx - 1)
    const int line0 = line_first - (f.lines - f.nb);
    const float* plane = dil + (long long)((f.rows_major ? 0 : 2) + (f.band - 1)) * n;
    ceiling_scan(plane, f, S.cols, line0, s_seg, out);
}

// grid (ceil((rows + cols) / 32), 1, hours), block (32, kCeilWarps): the ceiling plane
// of every daytime hour whose ray has at least kCeilMinSteps steps, from the
// dilated planes of ceiling_dilate_kernel.
static __global__ void __launch_bounds__(kCeilLanes * kCeilWarps) day_ray_ceiling_kernel(
    SolweigScene S, const SolweigHour* __restrict__ hours, const float* __restrict__ dil,
    float2* __restrict__ ceiling) {
    __shared__ float s_seg[kCeilWarps][kCeilLanes];
    const SolweigHour& h = hours[blockIdx.z];
    if (!h.daytime) return;
    ray_ceiling_block(S, reinterpret_cast<const int2*>(h.ray_dxdy), h.ray_dz, h.steps, dil,
                      ceiling + (long long)blockIdx.z * S.rows * S.cols, s_seg);
}

// The same for sky-patch rays: grid.z = patch - patch0 of a group of count
// patches; tables [patch][capacity] with lengths[patch] steps.
static __global__ void __launch_bounds__(kCeilLanes * kCeilWarps) patch_ray_ceiling_kernel(
    SolweigScene S, const int2* __restrict__ rays, const double* __restrict__ dz,
    const int32_t* __restrict__ lengths, int capacity, int patch0, int count, const float* __restrict__ dil,
    float2* __restrict__ ceiling) {
    __shared__ float s_seg[kCeilWarps][kCeilLanes];
    const int j = blockIdx.z, patch = patch0 + j;
    if (j >= count) return;
    const long long base = (long long)patch * capacity;
    ray_ceiling_block(S, rays + base, dz + base, lengths[patch], dil,
                      ceiling + (long long)j * S.rows * S.cols, s_seg);
}

}  // namespace solweig
