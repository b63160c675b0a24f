// Dyadic intervals on the host: the dissection of a real interval into
// maximal dyadic pieces used by every stream query.
//
// Restated from intervals/src/dyadic_interval.cpp:47-224 (the DyadicInterval
// constructors, expand/shrink/flip/advance, contains and aligned, and
// to_dyadic_intervals) and intervals/src/dyadic.cpp:74-101 (rebase).  For the
// clopen intervals that every query uses, each step of the reference's walk
// reduces to integer operations on the multiplier k of k / 2^p:
//   * expanding [k, k+1) / 2^p to its parent gives k >> 1 at power p - 1
//     (an odd k is first rounded down to the even one, rebase then halves);
//   * shrinking the parent to the contained end gives 2 (k >> 1); flipping
//     that even multiplier adds one, so the omitted end of the parent of an
//     odd k is k itself;
//   * [kb] at power pb contains [ke] at power pe >= pb exactly when
//     kb * 2^(pe - pb) equals ke rounded down to a multiple of 2^(pe - pb),
//     i.e. when kb == ke >> (pe - pb);
//   * an interval is "aligned" when it equals the left half of its parent,
//     compared as the reference compares intervals: both ends as doubles.
//     That is "k is even" whenever |k| < 2^53.
// The reference's walk, its iteration guard and its piece order are kept.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>

#include "common.cuh"

namespace rpyb {
namespace {

// x * 2^e, equal to std::ldexp(x, e): for |e| <= 1000 the factor 2^e is a
// normal double, and both round the exact product once
inline double scale2(double x, int32_t e)
{
    if (e < -1000 || e > 1000) return std::ldexp(x, e);
    const uint64_t bits = (uint64_t)(1023 + e) << 52;
    double f;
    std::memcpy(&f, &bits, sizeof f);
    return x * f;
}

// floor(k / 2^s) for s >= 0 (an arithmetic shift; beyond 63 bits only the
// sign remains)
inline int64_t shr(int64_t k, int32_t s) { return k >> std::min<int32_t>(s, 63); }

// [k, k+1) / 2^p equals [2 (k>>1), 2 (k>>1) + 1) / 2^p, both ends compared
// as doubles (dyadic_interval.cpp aligned(): the interval against the left
// half of its parent); the power of two scales both sides alike
inline bool aligned(int64_t k)
{
    const int64_t e = k & ~int64_t(1);
    return (double)k == (double)e && (double)(k + 1) == (double)(e + 1);
}

// The walks below with |k| < 2^52 throughout (so that "aligned" is "k is
// even"), without branches on the parity: it decides every step and is
// unpredictable.  Same steps, pieces and order as dissect_general.
int dissect_small(int64_t kb, int64_t ke, int32_t tol, int64_t* ko, int32_t* po)
{
    int32_t pb = tol, pe = tol;
    int nf = 0;
    while ((ke >> (pe - pb)) != kb) {
        const int64_t odd = kb & 1;
        ko[nf] = kb;
        po[nf] = pb;
        nf += (int)odd;
        kb = (kb >> 1) + odd;
        --pb;
    }
    int64_t back_k[64];
    int32_t back_p[64];
    int nb = 0;
    for (;;) {
        const int64_t nk = ke >> 1;
        const int32_t np = pe - 1;
        if (!(np >= pb && (nk >> (np - pb)) == kb)) break;
        back_k[nb] = 2 * nk;
        back_p[nb] = pe;
        nb += (int)(ke & 1);
        ke = nk;
        pe = np;
    }
    for (int i = 0; i < nb; ++i) {
        ko[nf + i] = back_k[nb - 1 - i];
        po[nf + i] = back_p[nb - 1 - i];
    }
    return nf + nb;
}

// to_dyadic_intervals (dyadic_interval.cpp:191-224) for a clopen interval at
// resolution tol; writes the pieces in order and returns their number
int dissect_general(int64_t kb, int64_t ke, int32_t tol, int64_t* ko, int32_t* po)
{
    constexpr int kGuard = 4 * 64;   // powers are bounded by the int64 range
    int32_t pb = tol, pe = tol;
    int nf = 0;
    // walk up from the included end; every unaligned interval on the way is
    // a piece, and the walk continues from the parent's right neighbour
    for (int guard = 0; shr(ke, pe - pb) != kb;) {
        if (!aligned(kb)) {
            ko[nf] = kb;
            po[nf] = pb;
            ++nf;
            kb = (kb >> 1) + 1;
        } else {
            kb >>= 1;
        }
        --pb;
        if (++guard > kGuard) break;
    }
    // walk up from the excluded end while the parent stays inside the
    // interval reached above; the left sibling of every unaligned interval
    // is a piece, and these come out in reverse walking order
    int64_t back_k[kGuard + 1];
    int32_t back_p[kGuard + 1];
    int nb = 0;
    for (int guard = 0;;) {
        const int64_t nk = ke >> 1;
        const int32_t np = pe - 1;
        if (!(np >= pb && shr(nk, np - pb) == kb)) break;
        if (!aligned(ke)) {
            back_k[nb] = 2 * nk;
            back_p[nb] = pe;
            ++nb;
        }
        ke = nk;
        pe = np;
        if (++guard > kGuard) break;
    }
    for (int i = 0; i < nb; ++i) {
        ko[nf + i] = back_k[nb - 1 - i];
        po[nf + i] = back_p[nb - 1 - i];
    }
    return nf + nb;
}

int dissect_walk(double inf, double sup, int32_t tol, int64_t* ko, int32_t* po)
{
    const int64_t kb = (int64_t)std::floor(scale2(inf, tol));
    const int64_t ke = (int64_t)std::floor(scale2(sup, tol));
    constexpr int64_t kSmall = int64_t(1) << 52;
    if (kb > -kSmall && kb < kSmall && ke > -kSmall && ke < kSmall)
        return dissect_small(kb, ke, tol, ko, po);
    return dissect_general(kb, ke, tol, ko, po);
}

int check_query(double inf, double sup, int32_t tol, int clopen)
{
    if (!clopen)
        return fail(RPYB_E_UNSUPPORTED, "only clopen intervals are supported (as in RoughPy)");
    if (!(inf <= sup)) return fail(RPYB_E_INVALID, "inf must not be larger than sup");
    if (tol < -60 || tol > 60) return fail(RPYB_E_INVALID, "resolution out of range");
    const double lim = std::ldexp(1.0, 60 - (tol > 0 ? tol : 0));
    if (!(std::fabs(inf) < lim && std::fabs(sup) < lim))
        return fail(RPYB_E_INVALID, "interval end too large for the resolution");
    return RPYB_OK;
}

}  // namespace

int dissect_clopen(double inf, double sup, int32_t tol, int64_t* k, int32_t* p)
{
    if (int rc = check_query(inf, sup, tol, 1)) return rc;
    return dissect_walk(inf, sup, tol, k, p);
}

}  // namespace rpyb

using namespace rpyb;

extern "C" {

RPYB_API int64_t rpyb_dyadic_dissect(double inf, double sup, int32_t tol, int clopen,
                                     int64_t* k, int32_t* p, int64_t cap)
{
    if (int rc = check_query(inf, sup, tol, clopen)) return rc;
    int64_t kb[kMaxDyadicPieces];
    int32_t pb[kMaxDyadicPieces];
    const int64_t n = dissect_walk(inf, sup, tol, kb, pb);
    for (int64_t i = 0; i < n && i < cap; ++i) {
        if (k) k[i] = kb[i];
        if (p) p[i] = pb[i];
    }
    return n;
}

RPYB_API int rpyb_dyadic_dissect_batch(int64_t n, const double* inf, const double* sup,
                                       const int32_t* tol, int clopen, int64_t* k, int32_t* p,
                                       int64_t cap, int64_t* offsets)
{
    if (n < 0) return fail(RPYB_E_INVALID, "negative number of intervals");
    if (n > 0 && (!inf || !sup || !tol || !offsets))
        return fail(RPYB_E_INVALID, "null pointer");
    int64_t kb[kMaxDyadicPieces];
    int32_t pb[kMaxDyadicPieces];
    int64_t pos = 0;
    offsets[0] = 0;
    for (int64_t q = 0; q < n; ++q) {
        if (int rc = check_query(inf[q], sup[q], tol[q], clopen)) return rc;
        const int np = dissect_walk(inf[q], sup[q], tol[q], kb, pb);
        if (pos + np > cap) return fail(RPYB_E_NOMEM, "dissection output capacity exceeded");
        std::memcpy(k + pos, kb, (size_t)np * sizeof(int64_t));
        std::memcpy(p + pos, pb, (size_t)np * sizeof(int32_t));
        pos += np;
        offsets[q + 1] = pos;
    }
    return RPYB_OK;
}

}  // extern "C"
