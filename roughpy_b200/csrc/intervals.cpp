// Dyadic intervals on the host: the dissection of a real interval into
// maximal dyadic pieces used by every stream query.
//
// Restated from intervals/src/dyadic_interval.cpp:47-224 and
// intervals/src/dyadic.cpp:74-101 (rebase) with the same integer arithmetic,
// including its corner cases: clopen intervals round the included end down,
// opencl intervals round it up; `expand` produces a clopen interval; an
// interval is "aligned" when it equals the left half of its parent compared
// as a clopen interval.
#include <cmath>
#include <cstdint>
#include <vector>

#include "common.cuh"

namespace rpyb {
namespace {

struct Dyadic {
    int64_t k = 0;   // multiplier
    int32_t p = 0;   // power: value k / 2^p
};

inline int64_t pow2(int32_t e) { return int64_t(1) << e; }

inline int64_t mod(int64_t a, int64_t b)
{
    const int64_t r = a % b;
    return (r < 0) ? (r + (b < 0 ? -b : b)) : r;
}

// dyadic.cpp:74-101
bool rebase(Dyadic& d, int32_t res)
{
    if (d.k == 0) {
        d.p = res;
        return true;
    }
    if (res >= d.p) {
        d.k = d.k * pow2(res - d.p);
        d.p = res;
        return true;
    }
    int32_t r = d.p - res;
    while (d.k % pow2(r) != 0) --r;
    d.k /= pow2(r);
    d.p -= r;
    return res == d.p;
}

struct DyadicInterval {
    Dyadic d;
    bool clopen = true;

    int64_t unit() const { return clopen ? 1 : -1; }

    // DyadicInterval(Dyadic, resolution, type): dyadic_interval.cpp:47-59
    static DyadicInterval from_dyadic(Dyadic dy, int32_t res, bool clopen)
    {
        DyadicInterval di;
        di.d = dy;
        di.clopen = clopen;
        if (!rebase(di.d, res)) {
            const int64_t k1 = di.d.k;
            const int64_t one = di.unit();
            const int64_t pw = pow2(di.d.p - res);
            di.d.k = one * (k1 * one - mod(k1 * one, pw));
            rebase(di.d, res);
        }
        return di;
    }

    // DyadicInterval(param_t, resolution, type): dyadic_interval.cpp:60-71
    static DyadicInterval from_value(double val, int32_t res, bool clopen)
    {
        DyadicInterval di;
        di.clopen = clopen;
        const double rescaled = std::ldexp(val, res);
        di.d.k = clopen ? (int64_t)std::floor(rescaled) : (int64_t)std::ceil(rescaled);
        di.d.p = res;
        return di;
    }

    double inf() const
    {
        const int64_t kk = clopen ? d.k : d.k + unit();
        return std::ldexp((double)kk, -d.p);
    }
    double sup() const
    {
        const int64_t kk = clopen ? d.k + unit() : d.k;
        return std::ldexp((double)kk, -d.p);
    }

    bool equals(const DyadicInterval& o) const
    {
        return clopen == o.clopen && inf() == o.inf() && sup() == o.sup();
    }

    DyadicInterval shrink_to_contained_end() const { return from_dyadic(d, d.p + 1, clopen); }
    DyadicInterval& flip()
    {
        if ((d.k % 2) == 0) d.k += unit();
        else d.k -= unit();
        return *this;
    }
    DyadicInterval shrink_to_omitted_end() const
    {
        DyadicInterval t = shrink_to_contained_end();
        t.flip();
        return t;
    }
    // expand_interval: a clopen interval one power coarser
    DyadicInterval& expand(int32_t arg = 1)
    {
        *this = from_dyadic(d, d.p - arg, true);
        return *this;
    }
    DyadicInterval& advance()
    {
        d.k += unit();
        return *this;
    }
    bool contains_dyadic(const DyadicInterval& o) const
    {
        if (o.clopen != clopen) return false;
        if (o.d.p >= d.p) {
            const int64_t one = unit();
            const int64_t pw = pow2(o.d.p - d.p);
            const int64_t shifted = d.k * pw;
            const int64_t aligned = one * (o.d.k * one - mod(o.d.k * one, pw));
            return shifted == aligned;
        }
        return false;
    }
    bool aligned() const
    {
        const DyadicInterval parent = from_dyadic(d, d.p - 1, clopen);
        const DyadicInterval back = from_dyadic(parent.d, d.p, true);
        return equals(back);
    }
};

// dyadic_interval.cpp:191-224
std::vector<DyadicInterval> to_dyadic_intervals(double inf, double sup, int32_t tol, bool clopen)
{
    std::vector<DyadicInterval> front, back;
    const double included = clopen ? inf : sup;
    const double excluded = clopen ? sup : inf;
    DyadicInterval begin = DyadicInterval::from_value(included, tol, clopen);
    DyadicInterval end = DyadicInterval::from_value(excluded, tol, clopen);

    int guard = 0;
    while (!begin.contains_dyadic(end)) {
        DyadicInterval next = begin;
        next.expand();
        if (!begin.aligned()) {
            front.push_back(next.shrink_to_omitted_end());
            next.advance();
        }
        begin = next;
        if (++guard > 4 * 64) break;   // powers are bounded by the int64 range
    }
    // the pieces found walking down from `end` are inserted in front of the
    // previous insertion point, i.e. they come out in reverse walking order
    DyadicInterval next = end;
    guard = 0;
    while (begin.contains_dyadic(next.expand())) {
        if (!end.aligned()) back.push_back(next.shrink_to_contained_end());
        end = next;
        if (++guard > 4 * 64) break;
    }
    std::vector<DyadicInterval> out = front;
    for (auto it = back.rbegin(); it != back.rend(); ++it) out.push_back(*it);
    if (!clopen) {
        std::vector<DyadicInterval> rev(out.rbegin(), out.rend());
        return rev;
    }
    return out;
}

}  // namespace
}  // namespace rpyb

using namespace rpyb;

extern "C" {

static int check_query(double inf, double sup, int32_t tol, int clopen)
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

RPYB_API int64_t rpyb_dyadic_dissect(double inf, double sup, int32_t tol, int clopen,
                                     int64_t* k, int32_t* p, int64_t cap)
{
    if (int rc = check_query(inf, sup, tol, clopen)) return rc;
    const auto pieces = to_dyadic_intervals(inf, sup, tol, clopen != 0);
    const int64_t n = (int64_t)pieces.size();
    for (int64_t i = 0; i < n && i < cap; ++i) {
        if (k) k[i] = pieces[i].d.k;
        if (p) p[i] = pieces[i].d.p;
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
    int64_t pos = 0;
    offsets[0] = 0;
    for (int64_t q = 0; q < n; ++q) {
        if (int rc = check_query(inf[q], sup[q], tol[q], clopen)) return rc;
        const auto pieces = to_dyadic_intervals(inf[q], sup[q], tol[q], clopen != 0);
        for (const auto& piece : pieces) {
            if (pos >= cap) return fail(RPYB_E_NOMEM, "dissection output capacity exceeded");
            k[pos] = piece.d.k;
            p[pos] = piece.d.p;
            ++pos;
        }
        offsets[q + 1] = pos;
    }
    return RPYB_OK;
}

}  // extern "C"
