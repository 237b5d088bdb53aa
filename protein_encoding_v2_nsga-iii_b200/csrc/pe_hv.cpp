// pe_hv.cpp -- exact hypervolume for the quality metric of src/main.cu:820-858
// (the reference pipes its normalised objectives to a prebuilt `hv` binary).
//
// WFG algorithm (While, Bradstreet, Barone, "A Fast Way of Calculating Exact
// Hypervolumes", IEEE TEC 16(1), 2012): hv(S) = sum_k [ inclhv(s_k) -
// hv(nd(limit(S_{>k}, s_k))) ], with a sweep for two objectives.  Minimisation,
// reference point r; points not strictly inside r contribute nothing.
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

// non-dominated subset, one copy of duplicates
int nondominated(Pts &p, int n, int d)
{
    std::vector<char> keep(n, 1);
    for (int i = 0; i < n; i++) {
        if (!keep[i]) continue;
        for (int j = 0; j < n; j++) {
            if (i == j || !keep[j]) continue;
            if (weakly_dominates(&p[(size_t)j * d], &p[(size_t)i * d], d)) {
                keep[i] = 0;
                break;
            }
        }
    }
    int out = 0;
    for (int i = 0; i < n; i++)
        if (keep[i]) {
            if (out != i) std::memmove(&p[(size_t)out * d], &p[(size_t)i * d], sizeof(double) * d);
            out++;
        }
    p.resize((size_t)out * d);
    return out;
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

double wfg(Pts p, int n, int d, const double *r);

double inclhv(const double *x, int d, const double *r)
{
    double v = 1.0;
    for (int k = 0; k < d; k++) v *= r[k] - x[k];
    return v;
}

double wfg(Pts p, int n, int d, const double *r)
{
    if (n == 0) return 0.0;
    if (d == 1) {
        double mn = p[0];
        for (int i = 1; i < n; i++) mn = std::min(mn, p[i]);
        return r[0] - mn;
    }
    if (d == 2) return hv2(p, n, r);
    // sort by the last objective, worst first, so limit sets shrink quickly
    std::vector<int> ord(n);
    for (int i = 0; i < n; i++) ord[i] = i;
    std::sort(ord.begin(), ord.end(), [&](int a, int b) { return p[(size_t)a * d + d - 1] > p[(size_t)b * d + d - 1]; });
    Pts q((size_t)n * d);
    for (int i = 0; i < n; i++) std::memcpy(&q[(size_t)i * d], &p[(size_t)ord[i] * d], sizeof(double) * d);
    double vol = 0.0;
    for (int k = 0; k < n; k++) {
        const double *pk = &q[(size_t)k * d];
        vol += inclhv(pk, d, r);
        int m = n - k - 1;
        if (m == 0) continue;
        Pts lim((size_t)m * d);
        for (int j = 0; j < m; j++)
            for (int c = 0; c < d; c++) lim[(size_t)j * d + c] = std::max(pk[c], q[(size_t)(k + 1 + j) * d + c]);
        int mm = nondominated(lim, m, d);
        vol -= wfg(std::move(lim), mm, d, r);
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
    *out = wfg(std::move(p), k, d, ref);
    return PE_OK;
}
