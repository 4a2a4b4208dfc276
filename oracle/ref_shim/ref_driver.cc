// C entry points around the reference's own CPU correlator - TEST INFRASTRUCTURE ONLY.
//
// Compiled (with the pyre stand-ins of oracle/ref_shim/include) together with the unmodified
// reference sources lib/libampcor/correlators/Sequential.cc, lib/libampcor/dom/SLC.cc and
// lib/libampcor/dom/Raster.cc into oracle/_ref/libampcor_ref.so by oracle/Makefile.  Only the
// tests and the reference arm of bench.py load it, to pin the FP64 oracle to the reference's own
// arithmetic and to time the reference's CPU path; the product never does.
//
// ampcor_ref_sequential() drives the reference exactly as its Python worker would
// (pkg/ampcor/correlators/Sequential.py, CUDA.py:45-58): two SLC rasters opened from raw
// complex64 files (SLC.icc:122-126), one Sequential worker (Sequential.cc:123-141), the chip and
// window slices of every pair added with addReferenceTile / addTargetTile (Sequential.icc:15-182),
// then adjust() (Sequential.cc:17-97).  adjust() keeps its correlation surfaces in the private
// member _correlation and returns nothing; it is read here through a pointer to that member
// obtained by an explicit template instantiation (which is exempt from access checking), so
// the reference's header stays as it is.  With threads > 1 the pairs are split into that many
// consecutive groups, each run by its own Sequential worker on its own thread (the reference's
// worker is single-threaded; the workers share nothing but the read-only rasters).
#include <portinfo>

#include <ampcor/correlators.h>

#include <cstring>
#include <exception>
#include <thread>
#include <vector>

namespace {

using sequential_t = ampcor::correlators::Sequential;
using slc_t = ampcor::dom::slc_t;

struct correlation_member {
    using type = double* sequential_t::*;
    friend type member_of(correlation_member);
};

template <typename Tag, typename Tag::type M>
struct expose {
    friend typename Tag::type member_of(Tag) { return M; }
};

template struct expose<correlation_member, &sequential_t::_correlation>;

thread_local std::string g_error;

}  // namespace

extern "C" {

// The reference's coarse CPU correlation of `pairs` tile pairs.  ulhc: 4 int32 per pair (chip
// line, chip sample, window line, window sample); R, W: chip and window sizes; correlation:
// pairs x (W-R+1)^2 doubles, the surfaces of Sequential::adjust in pair order.  Returns 0, or -1
// with a message for ampcor_ref_error().
int ampcor_ref_sequential(const char* ref_path, long ref_lines, long ref_samples, const char* tgt_path,
                          long tgt_lines, long tgt_samples, const int* ulhc, long pairs, long R,
                          long W, double* correlation, int threads)
{
    try {
        const slc_t ref(ref_path, slc_t::shape_type{(size_t)ref_lines, (size_t)ref_samples});
        const slc_t tgt(tgt_path, slc_t::shape_type{(size_t)tgt_lines, (size_t)tgt_samples});
        const size_t C = (size_t)(W - R + 1);
        const slc_t::shape_type chip{(size_t)R, (size_t)R};
        const slc_t::shape_type window{(size_t)W, (size_t)W};
        if (threads < 1) threads = 1;
        if ((long)threads > pairs) threads = pairs > 0 ? (int)pairs : 1;
        std::vector<std::thread> pool;
        std::vector<std::string> errors((size_t)threads);
        auto run = [&](int t) {
            const long p0 = pairs * t / threads, p1 = pairs * (t + 1) / threads;
            if (p1 <= p0) return;
            try {
                sequential_t worker((size_t)(p1 - p0), chip, window);
                for (long p = p0; p < p1; ++p) {
                    const int* c = ulhc + 4 * p;
                    const slc_t::index_type rb{(size_t)c[0], (size_t)c[1]};
                    const slc_t::index_type tb{(size_t)c[2], (size_t)c[3]};
                    worker.addReferenceTile(ref, (size_t)(p - p0), ref.layout().slice(rb, rb + chip));
                    worker.addTargetTile(tgt, (size_t)(p - p0), tgt.layout().slice(tb, tb + window));
                }
                worker.adjust();
                const double* cor = worker.*member_of(correlation_member{});
                std::memcpy(correlation + (size_t)p0 * C * C, cor, sizeof(double) * (size_t)(p1 - p0) * C * C);
            } catch (const std::exception& e) {
                errors[(size_t)t] = e.what();
            }
        };
        for (int t = 1; t < threads; ++t) pool.emplace_back(run, t);
        run(0);
        for (auto& th : pool) th.join();
        for (auto& e : errors)
            if (!e.empty()) {
                g_error = e;
                return -1;
            }
        return 0;
    } catch (const std::exception& e) {
        g_error = e.what();
        return -1;
    }
}

// The reference's summed-area table (SumArea.icc:152-180) of a rows x cols grid of doubles, and
// its box sums (SumArea.icc:66-148) over the boxes [r0, r0 + h) x [c0, c0 + w) listed in boxes
// (4 longs each: r0, c0, h, w).
int ampcor_ref_sumarea(const double* a, long rows, long cols, double* table, const long* boxes,
                       long nboxes, double* sums)
{
    try {
        using grid_t = ampcor::correlators::heapgrid_t<2, double>;
        using sat_t = ampcor::correlators::sumarea_t<grid_t>;
        grid_t g{grid_t::layout_type{grid_t::shape_type{(size_t)rows, (size_t)cols}}};
        for (long i = 0; i < rows; ++i)
            for (long j = 0; j < cols; ++j) g[grid_t::index_type{(size_t)i, (size_t)j}] = a[i * cols + j];
        sat_t sat(g);
        for (long i = 0; i < rows; ++i)
            for (long j = 0; j < cols; ++j) table[i * cols + j] = sat[grid_t::index_type{(size_t)i, (size_t)j}];
        for (long k = 0; k < nboxes; ++k) {
            const long* b = boxes + 4 * k;
            const grid_t::index_type lo{(size_t)b[0], (size_t)b[1]};
            const grid_t::index_type hi{(size_t)(b[0] + b[2]), (size_t)(b[1] + b[3])};
            sums[k] = sat.sum(g.layout().slice(lo, hi));
        }
        return 0;
    } catch (const std::exception& e) {
        g_error = e.what();
        return -1;
    }
}

const char* ampcor_ref_error(void) { return g_error.c_str(); }

}  // extern "C"
