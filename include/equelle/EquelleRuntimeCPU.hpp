// equelle::EquelleRuntimeCPU -- the class Equelle-generated simulators call.
//
// Same public surface as sintefmath/equelle
// backends/serial/include/equelle/EquelleRuntimeCPU.hpp:35-134, so that the
// C++ the `ec` compiler emits (e.g. examples/app/out_heateq.cpp) compiles
// unchanged.  Every operation forwards to the C ABI in eqg.h; which library
// is linked (libeqg.so for the B200 device runtime, or the CPU oracle used
// by tests) decides where the work runs.  Host-side duties stay here, as in
// the reference: parameter access, input files (EquelleRuntimeCPU.cpp:
// 485-551, EquelleRuntimeCPU_impl.hpp:342-365) and output formatting
// (EquelleRuntimeCPU.cpp:449-482).
#pragma once

#include "equelle/ParameterGroup.hpp"
#include "equelle/equelleTypes.hpp"

#include <algorithm>
#include <cctype>
#include <charconv>
#include <cmath>
#include <condition_variable>
#include <deque>
#include <exception>
#include <cstdlib>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <iterator>
#include <map>
#include <mutex>
#include <sstream>
#include <string>
#include <thread>
#include <tuple>
#include <utility>
#include <vector>

namespace equelle {

namespace detail {

// The values of an input file: whitespace-separated text (the reference's
// format), or raw little-endian FP64 when the file name ends in ".f64"
// (large inputs, where parsing text would dominate a run).
inline std::vector<double> read_values(const std::string& filename)
{
    const bool binary = filename.size() > 4 && filename.compare(filename.size() - 4, 4, ".f64") == 0;
    if (binary) {
        std::ifstream is(filename.c_str(), std::ios::binary | std::ios::ate);
        if (!is) {
            throw std::runtime_error("Could not find file " + filename);
        }
        const std::streamsize bytes = is.tellg();
        if (bytes < 0 || bytes % 8 != 0) {
            throw std::runtime_error("File " + filename + " does not hold whole doubles");
        }
        std::vector<double> v((size_t)(bytes / 8));
        is.seekg(0);
        if (!v.empty() && !is.read(reinterpret_cast<char*>(v.data()), bytes)) {
            throw std::runtime_error("Could not read file " + filename);
        }
        return v;
    }
    std::ifstream is(filename.c_str(), std::ios::binary);
    if (!is) {
        throw std::runtime_error("Could not find file " + filename);
    }
    // the whole file, then std::from_chars over it: correctly rounded like
    // the stream's conversion, so the same values an istream reads, up to
    // the first token that is not a number, at a fraction of its cost per
    // value (a leading '+' is skipped; other forms go through strtod)
    std::string text((std::istreambuf_iterator<char>(is)), std::istreambuf_iterator<char>());
    std::vector<double> v;
    v.reserve(text.size() / 8);
    const char* p = text.c_str();
    const char* const end = p + text.size();
    for (;;) {
        while (p < end && std::isspace((unsigned char)*p)) ++p;
        if (p == end) break;
        double x = 0.0;
        const char* q = *p == '+' ? p + 1 : p;
        const auto r = std::from_chars(q, end, x);
        if (r.ec == std::errc()) {
            v.push_back(x);
            p = r.ptr;
            continue;
        }
        char* e = nullptr;
        x = std::strtod(p, &e);
        if (e == p) break;
        v.push_back(x);
        p = e;
    }
    return v;
}

}  // namespace detail

class EquelleRuntimeCPU {
public:
    /// Builds the grid from grid_dim, nx, ny, nz, dx, dy, dz and reads
    /// output_to_file, verbose, max_iter, abs_res_tol
    /// (EquelleRuntimeCPU.cpp:20-65).
    explicit EquelleRuntimeCPU(const Opm::ParameterGroup& param)
        : param_(param),
          output_to_file_(param.getDefault("output_to_file", false)),
          output_dir_(param.getDefault<std::string>("output_dir", "")),
          output_values_(param.getDefault<std::string>("output_values", "all") == "all"),
          output_last_(param.getDefault<std::string>("output_values", "all") == "last"),
          output_off_(param.getDefault<std::string>("output_values", "all") == "off"),
          verbose_(param.getDefault("verbose", 0))
    {
        const auto items = param.items();
        std::vector<const char*> keys, vals;
        for (const auto& kv : items) {
            keys.push_back(kv.first.c_str());
            vals.push_back(kv.second.c_str());
        }
        detail::check(eqg_runtime_create((int)items.size(), keys.data(), vals.data(), &rt_));
        detail::check(eqg_runtime_grid_info(rt_, &info_));
    }
    EquelleRuntimeCPU(const EquelleRuntimeCPU&) = delete;
    EquelleRuntimeCPU& operator=(const EquelleRuntimeCPU&) = delete;
    ~EquelleRuntimeCPU()
    {
        drainOutputs();
        if (!out_error_.empty()) {
            std::cerr << out_error_ << std::endl;
        }
        writeLastOutputs();
        eqg_runtime_destroy(rt_);
    }

    eqg_runtime* handle() const { return rt_; }
    const eqg_grid_info& gridInfo() const { return info_; }

    /** @name Topology (EquelleRuntimeCPU.cpp:80-314) */
    ///@{
    CollOfCell allCells() const { return builtinCells(EQG_ALL_CELLS); }
    CollOfCell boundaryCells() const { return builtinCells(EQG_BOUNDARY_CELLS); }
    CollOfCell interiorCells() const { return builtinCells(EQG_INTERIOR_CELLS); }
    CollOfFace allFaces() const { return builtinFaces(EQG_ALL_FACES); }
    CollOfFace boundaryFaces() const { return builtinFaces(EQG_BOUNDARY_FACES); }
    CollOfFace interiorFaces() const { return builtinFaces(EQG_INTERIOR_FACES); }
    CollOfCell firstCell(const CollOfFace& faces) const
    {
        eqg_set* out = nullptr;
        detail::check(eqg_first_cell(rt_, faces.handle(), &out));
        return CollOfCell(rt_, out);
    }
    CollOfCell secondCell(const CollOfFace& faces) const
    {
        eqg_set* out = nullptr;
        detail::check(eqg_second_cell(rt_, faces.handle(), &out));
        return CollOfCell(rt_, out);
    }
    CollOfScalar norm(const CollOfFace& faces) const { return measure(faces.handle()); }
    CollOfScalar norm(const CollOfCell& cells) const { return measure(cells.handle()); }
    CollOfScalar norm(const CollOfVector& vectors) const
    {
        CollOfScalar norm2 = vectors.col(0) * vectors.col(0);
        for (int d = 1; d < vectors.numCols(); ++d) {
            norm2 += vectors.col(d) * vectors.col(d);
        }
        return equelle::sqrt(norm2);
    }
    /// |x| with Jacobian sign(x) J (EquelleRuntimeCPU.cpp:241-254).
    CollOfScalar norm(const CollOfScalar& scalars) const { return detail::unary(EQG_ABS, scalars); }
    CollOfVector centroid(const CollOfFace& faces) const { return centroids(faces.handle()); }
    CollOfVector centroid(const CollOfCell& cells) const { return centroids(cells.handle()); }
    CollOfVector normal(const CollOfFace& faces) const
    {
        CollOfVector n(info_.dimensions);
        for (int d = 0; d < info_.dimensions; ++d) {
            eqg_coll* out = nullptr;
            detail::check(eqg_normal(rt_, faces.handle(), d, &out));
            n.col(d) = CollOfScalar(rt_, out);
        }
        return n;
    }
    ///@}

    /** @name Math (EquelleRuntimeCPU.cpp:317-391) */
    ///@{
    CollOfScalar sqrt(const CollOfScalar& x) const { return equelle::sqrt(x); }
    CollOfScalar dot(const CollOfVector& v1, const CollOfVector& v2) const
    {
        if (v1.numCols() != v2.numCols()) {
            throw std::logic_error("Non-matching dimension of Vectors for dot().");
        }
        if (v1.col(0).size() != v2.col(0).size()) {
            throw std::logic_error("Non-matching size of Vector collections for dot().");
        }
        CollOfScalar result = v1.col(0) * v2.col(0);
        for (int d = 1; d < info_.dimensions; ++d) {
            result += v1.col(d) * v2.col(d);
        }
        return result;
    }
    CollOfScalar gradient(const CollOfScalar& x) const { return stencil(eqg_gradient, x); }
    CollOfScalar negGradient(const CollOfScalar& x) const { return stencil(eqg_neg_gradient, x); }
    CollOfScalar divergence(const CollOfScalar& x) const { return stencil(eqg_divergence, x); }
    CollOfScalar interiorDivergence(const CollOfScalar& x) const { return stencil(eqg_interior_divergence, x); }
    CollOfBool isEmpty(const CollOfCell& cells) const { return emptyMask(cells.handle()); }
    CollOfBool isEmpty(const CollOfFace& faces) const { return emptyMask(faces.handle()); }

    /// Scalar Extend: a constant collection (EquelleRuntimeCPU_impl.hpp:15-20).
    template <class EntityColl>
    CollOfScalar operatorExtend(const Scalar data, const EntityColl& to_set)
    {
        eqg_coll* out = nullptr;
        detail::check(eqg_coll_constant(rt_, data, (int64_t)to_set.size(), &out));
        return CollOfScalar(rt_, out);
    }
    /// Extend with zeros (EquelleRuntimeCPU_impl.hpp:113-123).
    template <int C>
    CollOfScalar operatorExtend(const CollOfScalar& data, const EntityCollection<C>& from_set,
                                const EntityCollection<C>& to_set)
    {
        eqg_coll* out = nullptr;
        detail::check(eqg_extend(rt_, data.handle(), from_set.handle(), to_set.handle(), &out));
        return CollOfScalar(rt_, out);
    }
    template <int D, int C>
    EntityCollection<D> operatorExtend(const EntityCollection<D>& data, const EntityCollection<C>& from_set,
                                       const EntityCollection<C>& to_set)
    {
        eqg_set* out = nullptr;
        detail::check(eqg_set_extend(rt_, data.handle(), from_set.handle(), to_set.handle(), &out));
        return EntityCollection<D>(rt_, out);
    }
    /// Restriction to a subset, repeats allowed (EquelleRuntimeCPU_impl.hpp:127-141).
    template <int C>
    CollOfScalar operatorOn(const CollOfScalar& data, const EntityCollection<C>& from_set,
                            const EntityCollection<C>& to_set)
    {
        eqg_coll* out = nullptr;
        detail::check(eqg_on(rt_, data.handle(), from_set.handle(), to_set.handle(), &out));
        return CollOfScalar(rt_, out);
    }
    template <int D, int C>
    EntityCollection<D> operatorOn(const EntityCollection<D>& data, const EntityCollection<C>& from_set,
                                   const EntityCollection<C>& to_set)
    {
        eqg_set* out = nullptr;
        detail::check(eqg_set_on(rt_, data.handle(), from_set.handle(), to_set.handle(), &out));
        return EntityCollection<D>(rt_, out);
    }

    /// trinaryIf (EquelleRuntimeCPU_impl.hpp:145-207).
    CollOfScalar trinaryIf(const CollOfBool& predicate, const CollOfScalar& iftrue,
                           const CollOfScalar& iffalse) const
    {
        eqg_coll* out = nullptr;
        detail::check(eqg_select(rt_, predicate.handle(), iftrue.handle(), iffalse.handle(), &out));
        return CollOfScalar(rt_, out);
    }
    template <int C>
    EntityCollection<C> trinaryIf(const CollOfBool& predicate, const EntityCollection<C>& iftrue,
                                  const EntityCollection<C>& iffalse) const
    {
        eqg_set* out = nullptr;
        detail::check(eqg_set_select(rt_, predicate.handle(), iftrue.handle(), iffalse.handle(), &out));
        return EntityCollection<C>(rt_, out);
    }
    ///@}

    /** @name Reductions (EquelleRuntimeCPU.cpp:393-411) */
    ///@{
    Scalar minReduce(const CollOfScalar& x) const { return reduce(EQG_MIN, x); }
    Scalar maxReduce(const CollOfScalar& x) const { return reduce(EQG_MAX, x); }
    Scalar sumReduce(const CollOfScalar& x) const { return reduce(EQG_SUM, x); }
    Scalar prodReduce(const CollOfScalar& x) const { return reduce(EQG_PROD, x); }
    ///@}

    /** @name Solvers (EquelleRuntimeCPU_impl.hpp:210-339) */
    ///@{
    template <class ResidualFunctor>
    CollOfScalar newtonSolve(const ResidualFunctor& rescomp, const CollOfScalar& u_initialguess)
    {
        Trampoline<ResidualFunctor> ctx{&rescomp, rt_, nullptr};
        eqg_coll* out = nullptr;
        const int st = eqg_newton_solve(rt_, &Trampoline<ResidualFunctor>::call, &ctx, u_initialguess.handle(), &out);
        if (ctx.error) {
            std::rethrow_exception(ctx.error);
        }
        detail::check(st);
        return CollOfScalar(rt_, out);
    }

    /// Coupled solve of Num residuals in Num unknown collections: the
    /// unknowns are stacked into one primary variable, each residual sees
    /// the unstacked parts, and the residuals are stacked in the same order
    /// (EquelleRuntimeCPU_impl.hpp:282-339).  The reference accepts only
    /// Num == 2; any Num >= 1 works here.
    template <class... ResFuncs, class... Colls>
    std::tuple<Colls...> newtonSolveSystem(const std::tuple<ResFuncs...>& rescomp,
                                           const std::tuple<Colls...>& u_initialguess)
    {
        static_assert(sizeof...(ResFuncs) == sizeof...(Colls),
                      "Size of residual function and initial guess arrays must be identical.");
        return systemSolve(rescomp, u_initialguess, std::index_sequence_for<Colls...>{});
    }
    ///@}

    /** @name Output (EquelleRuntimeCPU.cpp:449-482) */
    ///@{
    void output(const String& tag, Scalar val) const
    {
        if (output_values_) {
            std::cout << tag << " = " << val << std::endl;
        }
    }
    /// The copy to the host runs on the device while the program goes on:
    /// a writer thread waits for it and writes the file, in call order (at
    /// most kPendingOutputs copies in flight); printed output waits for its
    /// copy, to keep its place among the program's other prints.
    /// Extensions for timing runs: output_values=none still copies each
    /// collection to the host but neither prints nor writes it;
    /// output_values=off does not copy it; output_values=last keeps the last
    /// collection of each tag and writes <output_dir><tag>-last.output
    /// (precision 17) when the runtime ends.  Every call also records two
    /// device clock marks, before and after starting the copy
    /// (outputMarks): for an explicit program, whose time steps are the
    /// intervals between its outputs.
    void output(const String& tag, const CollOfScalar& vals)
    {
        rethrowOutputError();
        int before = 0, after = 0;
        // values the runtime has deferred are computed here, before the
        // marks, so that they belong to the time step that made them
        detail::check(eqg_coll_evaluate(rt_, vals.handle()));
        detail::check(eqg_runtime_mark(rt_, &before));
        if (!output_off_) {
            int64_t ticket = 0;
            detail::check(eqg_output_begin(rt_, vals.handle(), &ticket));
            if (output_values_ && !output_to_file_) {
                writeTicket(tag, ticket);
            } else {
                enqueueOutput(tag, ticket);
            }
        }
        detail::check(eqg_runtime_mark(rt_, &after));
        auto it = output_marks_.find(tag);
        if (it == output_marks_.end()) {
            output_tags_.push_back(tag);
            it = output_marks_.emplace(tag, std::vector<std::pair<int, int>>()).first;
        }
        it->second.emplace_back(before, after);
    }
    /// Output tags in the order of their first output.
    const std::vector<String>& outputTags() const { return output_tags_; }
    /// (before, after) clock marks of every output of `tag`.
    const std::vector<std::pair<int, int>>& outputMarks(const String& tag) const
    {
        static const std::vector<std::pair<int, int>> none;
        auto it = output_marks_.find(tag);
        return it == output_marks_.end() ? none : it->second;
    }

private:
    static constexpr size_t kPendingOutputs = 8;

    void enqueueOutput(const String& tag, int64_t ticket)
    {
        std::unique_lock<std::mutex> lock(out_mutex_);
        if (!writer_.joinable()) {
            writer_ = std::thread([this] { writerLoop(); });
        }
        out_cv_.wait(lock, [this] { return out_queue_.size() < kPendingOutputs; });
        out_queue_.emplace_back(tag, ticket);
        out_cv_.notify_all();
    }
    void writerLoop()
    {
        for (;;) {
            std::pair<String, int64_t> item;
            {
                std::unique_lock<std::mutex> lock(out_mutex_);
                out_cv_.wait(lock, [this] { return !out_queue_.empty() || out_stop_; });
                if (out_queue_.empty()) {
                    return;
                }
                item = out_queue_.front();
            }
            try {
                writeTicket(item.first, item.second);
            } catch (const std::exception& e) {
                std::lock_guard<std::mutex> lock(out_mutex_);
                if (out_error_.empty()) {
                    out_error_ = e.what();
                }
            }
            {
                std::lock_guard<std::mutex> lock(out_mutex_);
                out_queue_.pop_front();
            }
            out_cv_.notify_all();
        }
    }
    void drainOutputs()
    {
        {
            std::lock_guard<std::mutex> lock(out_mutex_);
            out_stop_ = true;
        }
        out_cv_.notify_all();
        if (writer_.joinable()) {
            writer_.join();
        }
    }
    void rethrowOutputError()
    {
        std::lock_guard<std::mutex> lock(out_mutex_);
        if (!out_error_.empty()) {
            const std::string e = out_error_;
            out_error_.clear();
            throw std::runtime_error(e);
        }
    }
    void writeTicket(const String& tag, int64_t ticket)
    {
        struct Release {
            eqg_runtime* rt;
            int64_t ticket;
            ~Release() { eqg_output_release(rt, ticket); }
        } release{rt_, ticket};
        const double* v = nullptr;
        int64_t n = 0;
        detail::check(eqg_output_wait(rt_, ticket, &v, &n));
        writeValues(tag, v, v + n);
    }
    void writeValues(const String& tag, const double* first, const double* last)
    {
        if (output_last_) {
            last_output_[tag].assign(first, last);
            return;
        }
        if (!output_values_) {
            return;
        }
        if (output_to_file_) {
            int count = 0;
            auto it = outputcount_.find(tag);
            if (it == outputcount_.end()) {
                outputcount_[tag] = 1;
            } else {
                count = it->second++;
            }
            std::ostringstream fname;
            fname << output_dir_ << tag << "-" << std::setw(5) << std::setfill('0') << count << ".output";
            std::ofstream file(fname.str().c_str());
            if (!file) {
                throw std::runtime_error("Failed to open " + fname.str());
            }
            file.precision(16);
            std::copy(first, last, std::ostream_iterator<double>(file, "\n"));
        } else {
            std::cout << tag << " =\n";
            for (const double* p = first; p != last; ++p) {
                std::cout << std::setw(15) << std::left << *p << " ";
            }
            std::cout << std::endl;
        }
    }

public:
    ///@}

    /** @name Input (EquelleRuntimeCPU.cpp:485-551, _impl.hpp:342-365) */
    ///@{
    Scalar inputScalarWithDefault(const String& name, const Scalar default_value)
    {
        return param_.getDefault(name, default_value);
    }
    CollOfFace inputDomainSubsetOf(const String& name, const CollOfFace& superset)
    {
        return inputSubset<1>(name, superset, "faces");
    }
    CollOfCell inputDomainSubsetOf(const String& name, const CollOfCell& superset)
    {
        return inputSubset<0>(name, superset, "cells");
    }
    template <class SomeCollection>
    CollOfScalar inputCollectionOfScalar(const String& name, const SomeCollection& coll)
    {
        const int size = (int)coll.size();
        const bool from_file = param_.getDefault(name + "_from_file", false);
        eqg_coll* out = nullptr;
        if (from_file) {
            const String filename = param_.get<String>(name + "_filename");
            const std::vector<double> data = detail::read_values(filename);
            if (int(data.size()) != size) {
                throw std::runtime_error("Unexpected size of input data for " + name + " in file " + filename);
            }
            detail::check(eqg_coll_from_host(rt_, data.data(), (int64_t)size, &out));
        } else {
            detail::check(eqg_coll_constant(rt_, param_.get<double>(name), (int64_t)size, &out));
        }
        return CollOfScalar(rt_, out);
    }
    SeqOfScalar inputSequenceOfScalar(const String& name)
    {
        const String filename = param_.get<String>(name + "_filename");
        std::ifstream is(filename.c_str());
        if (!is) {
            throw std::runtime_error("Could not find file " + filename);
        }
        std::istream_iterator<Scalar> beg(is);
        std::istream_iterator<Scalar> end;
        return SeqOfScalar(beg, end);
    }
    ///@}

    void ensureGridDimensionMin(const int minimum_grid_dimension) const
    {
        if (info_.dimensions < minimum_grid_dimension) {
            std::ostringstream os;
            os << "Equelle simulator requires minimum " << minimum_grid_dimension << " dimensions, but grid only has "
               << info_.dimensions << " dimensions.";
            throw std::runtime_error(os.str());
        }
    }

private:
    void writeLastOutputs()
    {
        for (const auto& kv : last_output_) {
            std::ofstream file((output_dir_ + kv.first + "-last.output").c_str());
            file.precision(17);
            std::copy(kv.second.begin(), kv.second.end(), std::ostream_iterator<double>(file, "\n"));
        }
    }

    template <class F>
    struct Trampoline {
        const F* f;
        eqg_runtime* rt;
        std::exception_ptr error;
        static int call(void* user, const eqg_coll* u, eqg_coll** residual)
        {
            auto* self = static_cast<Trampoline*>(user);
            try {
                CollOfScalar uu = CollOfScalar::borrow(self->rt, u);
                CollOfScalar r = (*self->f)(uu);
                *residual = r.release();
                return 0;
            } catch (...) {
                self->error = std::current_exception();
                return 1;
            }
        }
    };

    CollOfCell builtinCells(int which) const
    {
        eqg_set* out = nullptr;
        detail::check(eqg_set_builtin(rt_, which, &out));
        return CollOfCell(rt_, out);
    }
    CollOfFace builtinFaces(int which) const
    {
        eqg_set* out = nullptr;
        detail::check(eqg_set_builtin(rt_, which, &out));
        return CollOfFace(rt_, out);
    }
    CollOfScalar measure(const eqg_set* s) const
    {
        eqg_coll* out = nullptr;
        detail::check(eqg_measure(rt_, s, &out));
        return CollOfScalar(rt_, out);
    }
    CollOfVector centroids(const eqg_set* s) const
    {
        CollOfVector c(info_.dimensions);
        for (int d = 0; d < info_.dimensions; ++d) {
            eqg_coll* out = nullptr;
            detail::check(eqg_centroid(rt_, s, d, &out));
            c.col(d) = CollOfScalar(rt_, out);
        }
        return c;
    }
    CollOfBool emptyMask(const eqg_set* s) const
    {
        eqg_mask* out = nullptr;
        detail::check(eqg_set_is_empty(rt_, s, &out));
        return CollOfBool(rt_, out);
    }
    CollOfScalar stencil(int (*fn)(eqg_runtime*, const eqg_coll*, eqg_coll**), const CollOfScalar& x) const
    {
        eqg_coll* out = nullptr;
        detail::check(fn(rt_, x.handle(), &out));
        return CollOfScalar(rt_, out);
    }
    Scalar reduce(int op, const CollOfScalar& x) const
    {
        double r = 0.0;
        detail::check(eqg_reduce(rt_, op, x.handle(), &r));
        return r;
    }
    CollOfScalar spanSubset(const CollOfScalar& u, int64_t start, int64_t num) const
    {
        eqg_coll* out = nullptr;
        detail::check(eqg_span_subset(rt_, u.handle(), start, num, &out));
        return CollOfScalar(rt_, out);
    }
    CollOfScalar spanSuperset(const CollOfScalar& u, int64_t start, int64_t total) const
    {
        eqg_coll* out = nullptr;
        detail::check(eqg_span_superset(rt_, u.handle(), start, total, &out));
        return CollOfScalar(rt_, out);
    }

    template <int C>
    EntityCollection<C> inputSubset(const String& name, const EntityCollection<C>& superset, const char* what)
    {
        const String filename = param_.get<String>(name + "_filename");
        std::ifstream is(filename.c_str());
        if (!is) {
            throw std::runtime_error("Could not find file " + filename);
        }
        std::istream_iterator<int> beg(is);
        std::istream_iterator<int> end;
        std::vector<int32_t> data(beg, end);
        eqg_set* out = nullptr;
        detail::check(eqg_set_from_host(rt_, C == 0 ? EQG_CELLS : EQG_FACES, data.data(), (int64_t)data.size(), &out));
        EntityCollection<C> sub(rt_, out);
        int sorted = 0, included = 0;
        detail::check(eqg_set_check_subset(rt_, sub.handle(), superset.handle(), &sorted, &included));
        if (!sorted) {
            throw std::runtime_error(std::string("Input set of ") + what + " was not sorted in ascending order.");
        }
        if (!included) {
            throw std::runtime_error(std::string("Given ") + what + " are not in the assumed subset.");
        }
        return sub;
    }

    template <class F, class Parts, std::size_t... J>
    static CollOfScalar callWithParts(const F& f, const Parts& parts, std::index_sequence<J...>)
    {
        return f(parts[J]...);
    }

    template <class... ResFuncs, class... Colls, std::size_t... I>
    std::tuple<Colls...> systemSolve(const std::tuple<ResFuncs...>& rescomp, const std::tuple<Colls...>& u0,
                                     std::index_sequence<I...> seq)
    {
        constexpr std::size_t Num = sizeof...(Colls);
        const std::array<CollOfScalar, Num> init{{CollOfScalar(std::get<I>(u0))...}};
        std::array<int64_t, Num> start{}, num{};
        int64_t total = 0;
        for (std::size_t i = 0; i < Num; ++i) {
            start[i] = total;
            num[i] = init[i].size();
            total += num[i];
        }
        auto combined_rescomp = [&](const CollOfScalar& u) -> CollOfScalar {
            std::array<CollOfScalar, Num> parts;
            for (std::size_t i = 0; i < Num; ++i) {
                parts[i] = spanSubset(u, start[i], num[i]);
            }
            const std::array<CollOfScalar, Num> res{{callWithParts(std::get<I>(rescomp), parts, seq)...}};
            CollOfScalar result = spanSuperset(res[0], start[0], total);
            for (std::size_t i = 1; i < Num; ++i) {
                result += spanSuperset(res[i], start[i], total);
            }
            return result;
        };
        CollOfScalar combined_u0 = spanSuperset(init[0], start[0], total);
        for (std::size_t i = 1; i < Num; ++i) {
            combined_u0 += spanSuperset(init[i], start[i], total);
        }
        if (verbose_ > 0) {
            std::cout << "Done with setup of combined things." << std::endl;
        }
        const CollOfScalar combined_u = newtonSolve(combined_rescomp, combined_u0);
        return std::tuple<Colls...>(spanSubset(combined_u, start[I], num[I])...);
    }

    Opm::ParameterGroup param_;
    bool output_to_file_;
    std::string output_dir_;
    bool output_values_;
    bool output_last_;
    bool output_off_;
    std::map<String, std::vector<std::pair<int, int>>> output_marks_;
    std::vector<String> output_tags_;
    std::map<std::string, std::vector<double>> last_output_;
    int verbose_;
    eqg_runtime* rt_ = nullptr;
    eqg_grid_info info_{};
    std::map<std::string, int> outputcount_;
    // asynchronous outputs: queue of (tag, copy ticket) and its writer
    std::mutex out_mutex_;
    std::condition_variable out_cv_;
    std::deque<std::pair<std::string, int64_t>> out_queue_;
    std::thread writer_;
    bool out_stop_ = false;
    std::string out_error_;
};

}  // namespace equelle
