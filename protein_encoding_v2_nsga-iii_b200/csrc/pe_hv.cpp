// pe_hv.cpp -- exact hypervolume for the quality metric of src/main.cu:820-858
// (the reference pipes its normalised objectives to a prebuilt `hv` binary) and
// for the hypervolume-stall rule of served design jobs.
//
// Minimisation, reference point r; points not strictly inside r contribute
// nothing.  The volume is a sum of exclusive contributions along the last
// objective (the slicing step of WFG: While, Bradstreet, Barone, "A Fast Way of
// Calculating Exact Hypervolumes", IEEE TEC 16(1), 2012): with the points sorted
// by the last objective, worst first, the part of point k's box that no later
// point covers is (r_last - p_k,last) x [its (d-1)-volume minus the (d-1)-volume
// of the later points limited to p_k].
//   d = 2   one sweep;
//   d = 3   a z-sweep over a 2-D staircase (sorted vector, area kept incrementally);
//   d = 4   per point, a z-sweep over the later points limited to it, in a z order
//           computed once; the sweep stops as soon as the limited staircase
//           covers the whole xy box (a later point dominates it in x and y);
//   d >= 5  the slicing recursion with non-dominated filtering of limit sets.
#include <algorithm>
#include <cstdint>
#include <cstring>
#include <vector>

#include "../../include/pe_nsga3.h"

namespace {

using Pts = std::vector<double>;  // flat, d per point

bool weakly_dominates(const double *a, const double *b, int d)
{
    for (int k = 0; k < d; k++)
        if (a[k] > b[k]) return false;
    return true;
}

// non-dominated subset, one copy of duplicates: after a lexicographic sort a
// point can only be weakly dominated by an earlier one, so each point is checked
// against the points kept so far.
int nondominated(Pts &p, int n, int d)
{
    std::vector<int> ord(n);
    for (int i = 0; i < n; i++) ord[i] = i;
    std::sort(ord.begin(), ord.end(), [&](int a, int b) {
        return std::lexicographical_compare(&p[(size_t)a * d], &p[(size_t)a * d + d], &p[(size_t)b * d],
                                            &p[(size_t)b * d + d]);
    });
    Pts out;
    out.reserve((size_t)n * d);
    int kept = 0;
    for (int t = 0; t < n; t++) {
        const double *x = &p[(size_t)ord[t] * d];
        bool dom = false;
        for (int j = 0; j < kept && !dom; j++) dom = weakly_dominates(&out[(size_t)j * d], x, d);
        if (dom) continue;
        out.insert(out.end(), x, x + d);
        kept++;
    }
    p.swap(out);
    return kept;
}

double hv2(const Pts &p, int n, const double *r)
{
    std::vector<int> ord(n);
    for (int i = 0; i < n; i++) ord[i] = i;
    std::sort(ord.begin(), ord.end(), [&](int a, int b) { return p[2 * a] < p[2 * b]; });
    double vol = 0.0, miny = r[1];
    for (int t = 0; t < n; t++) {
        const double x = p[2 * ord[t]], y = p[2 * ord[t] + 1];
        miny = std::min(miny, y);
        double xn = t + 1 < n ? std::min(p[2 * ord[t + 1]], r[0]) : r[0];
        if (xn > x && miny < r[1]) vol += (xn - x) * (r[1] - miny);
    }
    return vol;
}

// 2-D non-dominated staircase: x ascending, y strictly descending; `area` is the
// region it dominates inside (rx, ry).
struct Staircase {
    struct P {
        double x, y;
    };
    std::vector<P> s;
    double rx = 0, ry = 0, area = 0;

    void reset(double rx_, double ry_)
    {
        s.clear();
        rx = rx_;
        ry = ry_;
        area = 0.0;
    }
    void insert(double x, double y)
    {
        size_t i = std::lower_bound(s.begin(), s.end(), x, [](const P &a, double v) { return a.x < v; }) - s.begin();
        if (i > 0 && s[i - 1].y <= y) return;                     // dominated from the left
        if (i < s.size() && s[i].x == x && s[i].y <= y) return;   // same x, lower y
        const double yl = i > 0 ? s[i - 1].y : ry;
        size_t j = i;
        while (j < s.size() && s[j].y >= y) j++;                  // points the new one dominates
        const double xnext = j < s.size() ? s[j].x : rx;
        double old = 0.0;
        if (i == j) {
            old = (xnext - x) * (ry - yl);
        } else {
            old = (s[i].x - x) * (ry - yl);
            for (size_t t = i; t < j; t++) old += ((t + 1 < j ? s[t + 1].x : xnext) - s[t].x) * (ry - s[t].y);
        }
        area += (xnext - x) * (ry - y) - old;
        if (j - i == 1) {
            s[i] = {x, y};
        } else {
            s.erase(s.begin() + i, s.begin() + j);
            s.insert(s.begin() + i, {x, y});
        }
    }
};

double hv3(const Pts &p, int n, const double *r)
{
    std::vector<int> ord(n);
    for (int i = 0; i < n; i++) ord[i] = i;
    std::sort(ord.begin(), ord.end(), [&](int a, int b) { return p[3 * a + 2] < p[3 * b + 2]; });
    Staircase st;
    st.reset(r[0], r[1]);
    double vol = 0.0, zprev = 0.0;
    for (int t = 0; t < n; t++) {
        const double *q = &p[3 * (size_t)ord[t]];
        if (t > 0) vol += st.area * (q[2] - zprev);
        zprev = q[2];
        st.insert(q[0], q[1]);
    }
    if (n > 0) vol += st.area * (r[2] - zprev);
    return vol;
}

double hv4(const Pts &p, int n, const double *r)
{
    // w order (last objective), worst first; z order for every sweep
    std::vector<int> byw(n), rank(n), byz(n);
    for (int i = 0; i < n; i++) byw[i] = byz[i] = i;
    std::sort(byw.begin(), byw.end(), [&](int a, int b) { return p[4 * a + 3] > p[4 * b + 3]; });
    for (int k = 0; k < n; k++) rank[byw[k]] = k;
    std::sort(byz.begin(), byz.end(), [&](int a, int b) { return p[4 * a + 2] < p[4 * b + 2]; });
    Staircase st;
    double vol = 0.0;
    for (int k = 0; k < n; k++) {
        const double *pk = &p[4 * (size_t)byw[k]];
        const double full = (r[0] - pk[0]) * (r[1] - pk[1]);
        // 3-D volume of pk's box not covered by later points: sweep z upward from pk.z
        st.reset(r[0], r[1]);
        double uncovered = 0.0, zprev = pk[2];
        bool covered = false;
        for (int t = 0; t < n && !covered; t++) {
            const int j = byz[t];
            if (rank[j] <= k) continue;
            const double *q = &p[4 * (size_t)j];
            const double z = std::max(pk[2], q[2]);
            if (z > zprev) {
                uncovered += (full - st.area) * (z - zprev);
                zprev = z;
            }
            const double x = std::max(pk[0], q[0]), y = std::max(pk[1], q[1]);
            if (x == pk[0] && y == pk[1]) covered = true;  // the rest of the box is covered
            else st.insert(x, y);
        }
        if (!covered) uncovered += (full - st.area) * (r[2] - zprev);
        vol += (r[3] - pk[3]) * uncovered;
    }
    return vol;
}

double inclhv(const double *x, int d, const double *r)
{
    double v = 1.0;
    for (int k = 0; k < d; k++) v *= r[k] - x[k];
    return v;
}

double hv(Pts p, int n, int d, const double *r)
{
    if (n == 0) return 0.0;
    if (d == 1) {
        double mn = p[0];
        for (int i = 1; i < n; i++) mn = std::min(mn, p[i]);
        return r[0] - mn;
    }
    if (d == 2) return hv2(p, n, r);
    if (d == 3) return hv3(p, n, r);
    if (d == 4) return hv4(p, n, r);
    // slicing along the last objective, worst first
    std::vector<int> ord(n);
    for (int i = 0; i < n; i++) ord[i] = i;
    std::sort(ord.begin(), ord.end(), [&](int a, int b) { return p[(size_t)a * d + d - 1] > p[(size_t)b * d + d - 1]; });
    Pts q((size_t)n * d);
    for (int i = 0; i < n; i++) std::memcpy(&q[(size_t)i * d], &p[(size_t)ord[i] * d], sizeof(double) * d);
    const int e = d - 1;
    double vol = 0.0;
    for (int k = 0; k < n; k++) {
        const double *pk = &q[(size_t)k * d];
        double excl = inclhv(pk, e, r);
        const int m = n - k - 1;
        if (m > 0) {
            Pts lim((size_t)m * e);
            for (int j = 0; j < m; j++)
                for (int c = 0; c < e; c++) lim[(size_t)j * e + c] = std::max(pk[c], q[(size_t)(k + 1 + j) * d + c]);
            const int mm = nondominated(lim, m, e);
            excl -= hv(std::move(lim), mm, e, r);
        }
        vol += (r[e] - pk[e]) * excl;
    }
    return vol;
}

}  // namespace

extern "C" int pe_hypervolume(const double *pts, int32_t n, int32_t d, const double *ref, double *out)
{
    if (!out || !ref || d < 1 || d > PE_MAX_OBJ || n < 0 || (n > 0 && !pts)) return PE_ERR_ARG;
    Pts p;
    p.reserve((size_t)n * d);
    int k = 0;
    for (int i = 0; i < n; i++) {
        bool inside = true;
        for (int c = 0; c < d; c++)
            if (!(pts[(size_t)i * d + c] < ref[c])) inside = false;
        if (!inside) continue;
        p.insert(p.end(), pts + (size_t)i * d, pts + (size_t)i * d + d);
        k++;
    }
    k = nondominated(p, k, d);
    *out = hv(std::move(p), k, d, ref);
    return PE_OK;
}
