// UTCI: the 6th-order regression polynomial of Broede et al. (2012) in air
// temperature Ta, 10-m wind va, D = Tmrt - Ta and vapour pressure Pa (kPa),
// src/kernels/utci.cu of the reference.  The published 210-term coefficient
// table must be identical everywhere; it is stored here in canonical exponent
// order (Pa outermost, then D, then va, then Ta).
//
// solweig_utci evaluates the full polynomial per pixel (per-pixel weather).
// For the common case of scalar weather per hour, solweig_utci_collapse (a
// host function) folds Ta, va and Pa into seven coefficients of a polynomial
// in D, which the hourly kernels evaluate by Horner's rule.
#include "common.cuh"

namespace solweig {

#define SOLWEIG_UTCI_TABLE \
    6.07562052E-01, -2.27712343E-02, 8.06470249E-04, -1.54271372E-04, -3.24651735E-06, \
    7.32602852E-08, 1.35959073E-09, -2.25836520E+00, 8.80326035E-02, 2.16844454E-03, \
    -1.53347087E-05, -5.72983704E-07, -2.55090145E-09, -7.51269505E-01, -4.08350271E-03, \
    -5.21670675E-05, 1.94544667E-06, 1.14099531E-08, 1.58137256E-01, -6.57263143E-05, \
    2.22697524E-07, -4.16117031E-08, -1.27762753E-02, 9.66891875E-06, 2.52785852E-09, \
    4.56306672E-04, -1.74202546E-07, -5.91491269E-06, 3.98374029E-01, 1.83945314E-04, \
    -1.73754510E-04, -7.60781159E-07, 3.77830287E-08, 5.43079673E-10, -2.00518269E-02, \
    8.92859837E-04, 3.45433048E-06, -3.77925774E-07, -1.69699377E-09, 1.69992415E-04, \
    -4.99204314E-05, 2.47417178E-07, 1.07596466E-08, 8.49242932E-05, 1.35191328E-06, \
    -6.21531254E-09, -4.99410301E-06, -1.89489258E-08, 8.15300114E-08, 7.55043090E-04, \
    -5.65095215E-05, -4.52166564E-07, 2.46688878E-08, 2.42674348E-10, 1.54547250E-04, \
    5.24110970E-06, -8.75874982E-08, -1.50743064E-09, -1.56236307E-05, -1.33895614E-07, \
    2.49709824E-09, 6.51711721E-07, 1.94960053E-09, -1.00361113E-08, -1.21206673E-05, \
    -2.18203660E-07, 7.51269482E-09, 9.79063848E-11, 1.25006734E-06, -1.81584736E-09, \
    -3.52197671E-10, -3.36514630E-08, 1.35908359E-10, 4.17032620E-10, -1.30369025E-09, \
    4.13908461E-10, 9.22652254E-12, -5.08220384E-09, -2.24730961E-11, 1.17139133E-10, \
    6.62154879E-10, 4.03863260E-13, 1.95087203E-12, -4.73602469E-12, 5.12733497E+00, \
    -3.12788561E-01, -1.96701861E-02, 9.99690870E-04, 9.51738512E-06, -4.66426341E-07, \
    5.48050612E-01, -3.30552823E-03, -1.64119440E-03, -5.16670694E-06, 9.52692432E-07, \
    -4.29223622E-02, 5.00845667E-03, 1.00601257E-06, -1.81748644E-06, -1.25813502E-03, \
    -1.79330391E-04, 2.34994441E-06, 1.29735808E-04, 1.29064870E-06, -2.28558686E-06, \
    -3.69476348E-02, 1.62325322E-03, -3.14279680E-05, 2.59835559E-06, -4.77136523E-08, \
    8.64203390E-03, -6.87405181E-04, -9.13863872E-06, 5.15916806E-07, -3.59217476E-05, \
    3.28696511E-05, -7.10542454E-07, -1.24382300E-05, -7.38584400E-09, 2.20609296E-07, \
    -7.32469180E-04, -1.87381964E-05, 4.80925239E-06, -8.75492040E-08, 2.77862930E-05, \
    -5.06004592E-06, 1.14325367E-07, 2.53016723E-06, -1.72857035E-08, -3.95079398E-08, \
    -3.59413173E-07, 7.04388046E-07, -1.89309167E-08, -4.79768731E-07, 7.96079978E-09, \
    1.62897058E-09, 3.94367674E-08, -1.18566247E-09, 3.34678041E-10, -1.15606447E-10, \
    -2.80626406E+00, 5.48712484E-01, -3.99428410E-03, -9.54009191E-04, 1.93090978E-05, \
    -3.08806365E-01, 1.16952364E-02, 4.95271903E-04, -1.90710882E-05, 2.10787756E-03, \
    -6.98445738E-04, 2.30109073E-05, 4.17856590E-04, -1.27043871E-05, -3.04620472E-06, \
    5.14507424E-02, -4.32510997E-03, 8.99281156E-05, -7.14663943E-07, -2.66016305E-04, \
    2.63789586E-04, -7.01199003E-06, -1.06823306E-04, 3.61341136E-06, 2.29748967E-07, \
    3.04788893E-04, -6.42070836E-05, 1.16257971E-06, 7.68023384E-06, -5.47446896E-07, \
    -3.59937910E-08, -4.36497725E-06, 1.68737969E-07, 2.67489271E-08, 3.23926897E-09, \
    -3.53874123E-02, -2.21201190E-01, 1.55126038E-02, -2.63917279E-04, 4.53433455E-02, \
    -4.32943862E-03, 1.45389826E-04, 2.17508610E-04, -6.66724702E-05, 3.33217140E-05, \
    -2.26921615E-03, 3.80261982E-04, -5.45314314E-09, -7.96355448E-04, 2.53458034E-05, \
    -6.31223658E-06, 3.02122035E-04, -4.77403547E-06, 1.73825715E-06, -4.09087898E-07, \
    6.14155345E-01, -6.16755931E-02, 1.33374846E-03, 3.55375387E-03, -5.13027851E-04, \
    1.02449757E-04, -1.48526421E-03, -4.11469183E-05, -6.80434415E-06, -9.77675906E-06, \
    8.82773108E-02, -3.01859306E-03, 1.04452989E-03, 2.47090539E-04, 1.48348065E-03

static const double kUtciHost[210] = {SOLWEIG_UTCI_TABLE};
__constant__ double kUtciDev[210] = {SOLWEIG_UTCI_TABLE};

// Hardy (1998) saturation vapour pressure over water, hPa.
__host__ __device__ inline double saturation_hpa(double ta) {
    const double tk = ta + 273.15;
    double es = 2.7150305 * log(tk);
    es += -2.8365744E3 / (tk * tk);
    es += -6.028076559E3 / tk;
    es += 1.954263612E1;
    es += -2.737830188E-2 * tk;
    es += 1.6261698E-5 * tk * tk;
    es += 7.0229056E-10 * tk * tk * tk;
    es += -1.8680009E-13 * tk * tk * tk * tk;
    return exp(es) * 0.01;
}

template <typename Table>
__host__ __device__ inline double utci_poly(const Table& c, double ta, double va, double d, double pa) {
    double pt[7], pv[7], pd[7], pp[7];
    pt[0] = pv[0] = pd[0] = pp[0] = 1.0;
    for (int i = 1; i < 7; ++i) {
        pt[i] = pt[i - 1] * ta;
        pv[i] = pv[i - 1] * va;
        pd[i] = pd[i - 1] * d;
        pp[i] = pp[i - 1] * pa;
    }
    double u = ta;
    int t = 0;
    for (int ip = 0; ip < 7; ++ip)
        for (int id = 0; id < 7 - ip; ++id)
            for (int iv = 0; iv < 7 - ip - id; ++iv)
                for (int it = 0; it < 7 - ip - id - iv; ++it)
                    u += c[t++] * pt[it] * pv[iv] * pd[id] * pp[ip];
    return u;
}

struct DevTable {
    __device__ double operator[](int i) const { return kUtciDev[i]; }
};

__global__ void __launch_bounds__(256) utci_kernel(const float* __restrict__ ta,
                                                   const float* __restrict__ rh,
                                                   const float* __restrict__ tmrt,
                                                   const float* __restrict__ va, int ta_s, int rh_s,
                                                   int va_s, float* __restrict__ out, long long n) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double t = ta[ta_s ? 0 : i], h = rh[rh_s ? 0 : i], w = va[va_s ? 0 : i];
    const double m = tmrt[i];
    if (t <= -999.0 || h <= -999.0 || w <= -999.0 || m <= -999.0) {
        out[i] = -999.0f;
        return;
    }
    const double pa = saturation_hpa(t) * h / 100.0 / 10.0;
    out[i] = (float)utci_poly(DevTable{}, t, w, m - t, pa);
}

// Scalar weather: UTCI(Tmrt) = sum_k c_k (Tmrt - Ta)^k by Horner's rule.
struct UtciPoly {
    double c[7];
    double ta;
    int valid;
};

__global__ void __launch_bounds__(256) utci_poly_kernel(UtciPoly poly, const float* __restrict__ tmrt,
                                                        float* __restrict__ out, long long n) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double m = tmrt[i];
    if (!poly.valid || m <= -999.0) {
        out[i] = -999.0f;
        return;
    }
    const double d = m - poly.ta;
    double u = poly.c[6];
#pragma unroll
    for (int k = 5; k >= 0; --k) u = u * d + poly.c[k];
    out[i] = (float)u;
}

}  // namespace solweig

using namespace solweig;

extern "C" int solweig_utci_collapse(double ta, double rh, double va, double* coefficients);

extern "C" int solweig_utci_scalar(double ta, double rh, double va, const float* tmrt, float* out,
                                   int64_t n, void* stream) {
    SOLWEIG_CHECK_ARG(tmrt && out && n >= 0, "solweig_utci_scalar: bad arguments");
    if (n == 0) return SOLWEIG_OK;
    UtciPoly poly{};
    poly.ta = ta;
    poly.valid = !(ta <= -999.0 || rh <= -999.0 || va <= -999.0);
    int rc = solweig_utci_collapse(ta, rh, va, poly.c);
    if (rc) return rc;
    utci_poly_kernel<<<blocks_for(n, 256), 256, 0, as_stream(stream)>>>(poly, tmrt, out, n);
    SOLWEIG_CHECK_LAUNCH("utci_poly_kernel");
    return SOLWEIG_OK;
}

extern "C" int solweig_utci_collapse(double ta, double rh, double va, double* coefficients) {
    SOLWEIG_CHECK_ARG(coefficients, "solweig_utci_collapse: null output");
    for (int i = 0; i < 7; ++i) coefficients[i] = 0.0;
    if (ta <= -999.0 || rh <= -999.0 || va <= -999.0) return SOLWEIG_OK;
    const double pa = saturation_hpa(ta) * rh / 100.0 / 10.0;
    double pt[7], pv[7], pp[7];
    pt[0] = pv[0] = pp[0] = 1.0;
    for (int i = 1; i < 7; ++i) {
        pt[i] = pt[i - 1] * ta;
        pv[i] = pv[i - 1] * va;
        pp[i] = pp[i - 1] * pa;
    }
    coefficients[0] = ta;
    int t = 0;
    for (int ip = 0; ip < 7; ++ip)
        for (int id = 0; id < 7 - ip; ++id)
            for (int iv = 0; iv < 7 - ip - id; ++iv)
                for (int it = 0; it < 7 - ip - id - iv; ++it)
                    coefficients[id] += kUtciHost[t++] * pt[it] * pv[iv] * pp[ip];
    return SOLWEIG_OK;
}

extern "C" int solweig_utci(const float* ta, const float* rh, const float* tmrt, const float* va,
                            int ta_scalar, int rh_scalar, int va_scalar, float* out, int64_t n,
                            void* stream) {
    SOLWEIG_CHECK_ARG(ta && rh && tmrt && va && out && n >= 0, "solweig_utci: bad arguments");
    if (n == 0) return SOLWEIG_OK;
    cudaStream_t st = as_stream(stream);
    utci_kernel<<<blocks_for(n, 256), 256, 0, st>>>(ta, rh, tmrt, va, ta_scalar, rh_scalar, va_scalar,
                                                    out, n);
    SOLWEIG_CHECK_LAUNCH("utci_kernel");
    return SOLWEIG_OK;
}
