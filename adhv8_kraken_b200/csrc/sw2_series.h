// Piecewise-linear boundary series and their average over a time step
// (sseries_set_values_average, src/structs/sseries.c:566-613): the boundary data a step sees is
// the mean of each series over the step, integrated exactly by trapezoids over the breakpoints
// inside the step, the end segments extrapolated linearly outside the table.  Host code (the
// continuous-batching engine evaluates the series of the solves it steps); plain C++, so the
// CPU tests compile it as it is.
#pragma once

#include <algorithm>
#include <vector>

namespace sw2 {

struct PwlSeries {
    std::vector<double> t, v;   // breakpoint times (ascending) and values
    double at(double tt) const {
        const size_t n = t.size();
        if (n == 1) return v[0];
        long i = (long)(std::upper_bound(t.begin(), t.end(), tt) - t.begin()) - 1;
        i = std::min(std::max(i, 0L), (long)n - 2);
        const double w = (tt - t[i]) / (t[i + 1] - t[i]);
        return v[i] + w * (v[i + 1] - v[i]);
    }
    double avg(double t1, double t2) const {
        if (t2 <= t1) return at(t1);
        double area = 0.0, a = t1;
        for (double x : t) {
            if (!(t1 < x && x < t2)) continue;
            area += 0.5 * (at(a) + at(x)) * (x - a);
            a = x;
        }
        area += 0.5 * (at(a) + at(t2)) * (t2 - a);
        return area / (t2 - t1);
    }
};

}  // namespace sw2
