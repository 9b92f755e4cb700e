// Value types of the Equelle runtime API, as generated simulators use them.
//
// Mirrors sintefmath/equelle backends/serial/include/equelle/equelleTypes.hpp
// (types :12-62, CollOfScalar :67-84, free operators :86-211, CollOfVector
// :215-316, CollType/makeArray :321-372, ResCompType :374-400, ESpan
// :407-498).  The collections here are handles to runtime-owned storage
// reached through the C ABI in eqg.h; values live wherever the linked
// library keeps them (device memory for libeqg.so).
#pragma once

#include "eqg.h"

#include <array>
#include <cassert>
#include <cstdint>
#include <functional>
#include <memory>
#include <stdexcept>
#include <string>
#include <tuple>
#include <utility>
#include <vector>

namespace equelle {

namespace detail {

inline void check(int status)
{
    if (status != EQG_OK) {
        throw std::runtime_error(eqg_last_error());
    }
}

inline eqg_runtime* pick(eqg_runtime* a, eqg_runtime* b)
{
    if (a) {
        return a;
    }
    if (b) {
        return b;
    }
    throw std::runtime_error("operation on an uninitialised collection");
}

}  // namespace detail

/// Codes for inner and outer boundaries.
enum Boundary { outer = -1, inner = -2 };

/// Topological entities (equelleTypes.hpp:15-24).
template <int Codim>
struct TopologicalEntity {
    TopologicalEntity() : index(-1) {}
    explicit TopologicalEntity(const int ind) : index(ind) {}
    int index;
    bool operator<(const TopologicalEntity& t) const { return index < t.index; }
    bool operator==(const TopologicalEntity& t) const { return index == t.index; }
};

typedef TopologicalEntity<0> Cell;
typedef TopologicalEntity<1> Face;

typedef double Scalar;
typedef bool Bool;
typedef std::string String;
typedef std::vector<Scalar> SeqOfScalar;

inline SeqOfScalar operator*(const SeqOfScalar& sos, Scalar s)
{
    SeqOfScalar res = sos;
    for (Scalar& r : res) {
        r *= s;
    }
    return res;
}
inline SeqOfScalar operator*(Scalar s, const SeqOfScalar& sos) { return sos * s; }
inline SeqOfScalar operator/(const SeqOfScalar& sos, Scalar s) { return sos * (Scalar(1) / s); }

/// A collection of cells (Codim 0) or faces (Codim 1).  The reference uses
/// std::vector<Cell>/std::vector<Face>; this handle offers the same read
/// access (size, operator[], iteration) through a host copy made on demand.
template <int Codim>
class EntityCollection {
public:
    typedef TopologicalEntity<Codim> value_type;

    EntityCollection() = default;
    EntityCollection(eqg_runtime* rt, eqg_set* adopted) : rt_(rt), h_(adopted) {}
    EntityCollection(const EntityCollection& o) : rt_(o.rt_), h_(o.h_), host_(o.host_)
    {
        eqg_set_retain(h_);
    }
    EntityCollection(EntityCollection&& o) noexcept : rt_(o.rt_), h_(o.h_), host_(std::move(o.host_))
    {
        o.h_ = nullptr;
    }
    EntityCollection& operator=(EntityCollection o) noexcept
    {
        std::swap(rt_, o.rt_);
        std::swap(h_, o.h_);
        std::swap(host_, o.host_);
        return *this;
    }
    ~EntityCollection() { eqg_set_release(h_); }

    size_t size() const
    {
        if (!h_) {
            return 0;
        }
        int64_t n = 0;
        detail::check(eqg_set_size(h_, &n));
        return (size_t)n;
    }
    bool empty() const { return size() == 0; }
    value_type operator[](size_t i) const { return value_type(hostIndices()[i]); }
    std::vector<value_type> toVector() const
    {
        std::vector<value_type> out;
        for (int v : hostIndices()) {
            out.emplace_back(v);
        }
        return out;
    }
    const std::vector<int>& hostIndices() const
    {
        if (!host_) {
            auto v = std::make_shared<std::vector<int>>(size());
            if (!v->empty()) {
                detail::check(eqg_set_to_host(h_, reinterpret_cast<int32_t*>(v->data())));
            }
            host_ = v;
        }
        return *host_;
    }

    eqg_set* handle() const { return h_; }
    eqg_runtime* runtime() const { return rt_; }

private:
    eqg_runtime* rt_ = nullptr;
    eqg_set* h_ = nullptr;
    mutable std::shared_ptr<std::vector<int>> host_;
};

typedef EntityCollection<0> CollOfCell;
typedef EntityCollection<1> CollOfFace;

/// Collection of booleans (the reference: Eigen::Array<bool, Dynamic, 1>).
class CollOfBool {
public:
    CollOfBool() = default;
    CollOfBool(eqg_runtime* rt, eqg_mask* adopted) : rt_(rt), h_(adopted) {}
    CollOfBool(const CollOfBool& o) : rt_(o.rt_), h_(o.h_) { eqg_mask_retain(h_); }
    CollOfBool(CollOfBool&& o) noexcept : rt_(o.rt_), h_(o.h_) { o.h_ = nullptr; }
    CollOfBool& operator=(CollOfBool o) noexcept
    {
        std::swap(rt_, o.rt_);
        std::swap(h_, o.h_);
        return *this;
    }
    ~CollOfBool() { eqg_mask_release(h_); }

    int size() const
    {
        if (!h_) {
            return 0;
        }
        int64_t n = 0;
        detail::check(eqg_mask_size(h_, &n));
        return (int)n;
    }
    std::vector<bool> toVector() const
    {
        std::vector<uint8_t> raw(size());
        if (!raw.empty()) {
            detail::check(eqg_mask_to_host(h_, raw.data()));
        }
        return std::vector<bool>(raw.begin(), raw.end());
    }
    bool operator[](int i) const { return toVector()[i]; }

    eqg_mask* handle() const { return h_; }
    eqg_runtime* runtime() const { return rt_; }

private:
    eqg_runtime* rt_ = nullptr;
    eqg_mask* h_ = nullptr;
};

inline CollOfBool logic(int op, const CollOfBool& a, const CollOfBool& b)
{
    eqg_mask* out = nullptr;
    eqg_runtime* rt = detail::pick(a.runtime(), b.runtime());
    detail::check(eqg_mask_logic(rt, op, a.handle(), b.handle(), &out));
    return CollOfBool(rt, out);
}
inline CollOfBool operator&&(const CollOfBool& a, const CollOfBool& b) { return logic(EQG_AND, a, b); }
inline CollOfBool operator||(const CollOfBool& a, const CollOfBool& b) { return logic(EQG_OR, a, b); }
inline CollOfBool operator!(const CollOfBool& a) { return logic(EQG_NOT, a, a); }

/// Collection Of Scalar: value plus, when it depends on a primary
/// variable, one sparse Jacobian block (Opm::AutoDiffBlock<double> in the
/// reference, equelleTypes.hpp:67-84).
class CollOfScalar {
public:
    CollOfScalar() = default;
    CollOfScalar(eqg_runtime* rt, eqg_coll* adopted) : rt_(rt), h_(adopted) {}
    CollOfScalar(const CollOfScalar& o) : rt_(o.rt_), h_(o.h_) { eqg_coll_retain(h_); }
    CollOfScalar(CollOfScalar&& o) noexcept : rt_(o.rt_), h_(o.h_) { o.h_ = nullptr; }
    CollOfScalar& operator=(CollOfScalar o) noexcept
    {
        std::swap(rt_, o.rt_);
        std::swap(h_, o.h_);
        return *this;
    }
    ~CollOfScalar() { eqg_coll_release(h_); }

    /// A new reference to a handle owned elsewhere.
    static CollOfScalar borrow(eqg_runtime* rt, const eqg_coll* h)
    {
        eqg_coll* m = const_cast<eqg_coll*>(h);
        eqg_coll_retain(m);
        return CollOfScalar(rt, m);
    }

    int size() const
    {
        if (!h_) {
            return 0;
        }
        int64_t n = 0;
        detail::check(eqg_coll_size(h_, &n));
        return (int)n;
    }
    /// Host copy of the values (AutoDiffBlock::value()).
    std::vector<double> value() const
    {
        std::vector<double> v(size());
        if (!v.empty()) {
            detail::check(eqg_coll_to_host(h_, v.data()));
        }
        return v;
    }
    bool hasJacobian() const
    {
        if (!h_) {
            return false;
        }
        int64_t r = 0, c = 0, nnz = 0;
        detail::check(eqg_coll_jacobian_info(h_, &r, &c, &nnz));
        return nnz >= 0;
    }

    eqg_coll* handle() const { return h_; }
    eqg_runtime* runtime() const { return rt_; }
    /// Gives up ownership of the handle (one reference).
    eqg_coll* release()
    {
        eqg_coll* h = h_;
        h_ = nullptr;
        return h;
    }

    CollOfScalar& operator+=(const CollOfScalar& rhs);

private:
    eqg_runtime* rt_ = nullptr;
    eqg_coll* h_ = nullptr;
};

namespace detail {

inline CollOfScalar binary(int op, const CollOfScalar& a, const CollOfScalar& b)
{
    eqg_runtime* rt = pick(a.runtime(), b.runtime());
    eqg_coll* out = nullptr;
    check(eqg_binary(rt, op, a.handle(), b.handle(), &out));
    return CollOfScalar(rt, out);
}

inline CollOfScalar binaryScalar(int op, const CollOfScalar& a, Scalar s, bool scalar_left)
{
    eqg_runtime* rt = pick(a.runtime(), nullptr);
    eqg_coll* out = nullptr;
    check(eqg_binary_scalar(rt, op, a.handle(), s, scalar_left ? 1 : 0, &out));
    return CollOfScalar(rt, out);
}

inline CollOfScalar unary(int op, const CollOfScalar& a)
{
    eqg_runtime* rt = pick(a.runtime(), nullptr);
    eqg_coll* out = nullptr;
    check(eqg_unary(rt, op, a.handle(), &out));
    return CollOfScalar(rt, out);
}

inline CollOfBool compare(int op, const CollOfScalar& a, const CollOfScalar& b)
{
    eqg_runtime* rt = pick(a.runtime(), b.runtime());
    eqg_mask* out = nullptr;
    check(eqg_compare(rt, op, a.handle(), b.handle(), &out));
    return CollOfBool(rt, out);
}

inline CollOfBool compareScalar(int op, const CollOfScalar& a, Scalar s, bool scalar_left)
{
    eqg_runtime* rt = pick(a.runtime(), nullptr);
    eqg_mask* out = nullptr;
    check(eqg_compare_scalar(rt, op, a.handle(), s, scalar_left ? 1 : 0, &out));
    return CollOfBool(rt, out);
}

}  // namespace detail

inline CollOfScalar operator+(const CollOfScalar& a, const CollOfScalar& b) { return detail::binary(EQG_ADD, a, b); }
inline CollOfScalar operator-(const CollOfScalar& a, const CollOfScalar& b) { return detail::binary(EQG_SUB, a, b); }
inline CollOfScalar operator*(const CollOfScalar& a, const CollOfScalar& b) { return detail::binary(EQG_MUL, a, b); }
inline CollOfScalar operator/(const CollOfScalar& a, const CollOfScalar& b) { return detail::binary(EQG_DIV, a, b); }

inline CollOfScalar operator+(const CollOfScalar& a, Scalar s) { return detail::binaryScalar(EQG_ADD, a, s, false); }
inline CollOfScalar operator+(Scalar s, const CollOfScalar& a) { return detail::binaryScalar(EQG_ADD, a, s, true); }
inline CollOfScalar operator-(const CollOfScalar& a, Scalar s) { return detail::binaryScalar(EQG_SUB, a, s, false); }
inline CollOfScalar operator-(Scalar s, const CollOfScalar& a) { return detail::binaryScalar(EQG_SUB, a, s, true); }
inline CollOfScalar operator*(const CollOfScalar& a, Scalar s) { return detail::binaryScalar(EQG_MUL, a, s, false); }
inline CollOfScalar operator*(Scalar s, const CollOfScalar& a) { return detail::binaryScalar(EQG_MUL, a, s, true); }
/// x / s (equelleTypes.hpp:99-102) and s / x (:93-96).
inline CollOfScalar operator/(const CollOfScalar& a, Scalar s) { return detail::binaryScalar(EQG_DIV, a, s, false); }
inline CollOfScalar operator/(Scalar s, const CollOfScalar& a) { return detail::binaryScalar(EQG_DIV, a, s, true); }
/// Unary minus (equelleTypes.hpp:87-90).
inline CollOfScalar operator-(const CollOfScalar& a) { return detail::unary(EQG_NEG, a); }

inline CollOfScalar& CollOfScalar::operator+=(const CollOfScalar& rhs)
{
    *this = *this + rhs;
    return *this;
}

/// Comparisons (equelleTypes.hpp:104-192) act on values only.
inline CollOfBool operator<(const CollOfScalar& x, const CollOfScalar& y) { return detail::compare(EQG_LT, x, y); }
inline CollOfBool operator<=(const CollOfScalar& x, const CollOfScalar& y) { return detail::compare(EQG_LE, x, y); }
inline CollOfBool operator>(const CollOfScalar& x, const CollOfScalar& y) { return detail::compare(EQG_GT, x, y); }
inline CollOfBool operator>=(const CollOfScalar& x, const CollOfScalar& y) { return detail::compare(EQG_GE, x, y); }
inline CollOfBool operator==(const CollOfScalar& x, const CollOfScalar& y) { return detail::compare(EQG_EQ, x, y); }
inline CollOfBool operator!=(const CollOfScalar& x, const CollOfScalar& y) { return detail::compare(EQG_NE, x, y); }
inline CollOfBool operator<(const CollOfScalar& x, Scalar s) { return detail::compareScalar(EQG_LT, x, s, false); }
inline CollOfBool operator<(Scalar s, const CollOfScalar& x) { return detail::compareScalar(EQG_LT, x, s, true); }
inline CollOfBool operator<=(const CollOfScalar& x, Scalar s) { return detail::compareScalar(EQG_LE, x, s, false); }
inline CollOfBool operator<=(Scalar s, const CollOfScalar& x) { return detail::compareScalar(EQG_LE, x, s, true); }
inline CollOfBool operator>(const CollOfScalar& x, Scalar s) { return detail::compareScalar(EQG_GT, x, s, false); }
inline CollOfBool operator>(Scalar s, const CollOfScalar& x) { return detail::compareScalar(EQG_GT, x, s, true); }
inline CollOfBool operator>=(const CollOfScalar& x, Scalar s) { return detail::compareScalar(EQG_GE, x, s, false); }
inline CollOfBool operator>=(Scalar s, const CollOfScalar& x) { return detail::compareScalar(EQG_GE, x, s, true); }
inline CollOfBool operator==(const CollOfScalar& x, Scalar s) { return detail::compareScalar(EQG_EQ, x, s, false); }
inline CollOfBool operator==(Scalar s, const CollOfScalar& x) { return detail::compareScalar(EQG_EQ, x, s, true); }
inline CollOfBool operator!=(const CollOfScalar& x, Scalar s) { return detail::compareScalar(EQG_NE, x, s, false); }
inline CollOfBool operator!=(Scalar s, const CollOfScalar& x) { return detail::compareScalar(EQG_NE, x, s, true); }

/// sqrt with d(sqrt(x)) = 1/(2 sqrt(x)) dx (equelleTypes.hpp:195-211).
inline CollOfScalar sqrt(const CollOfScalar& x) { return detail::unary(EQG_SQRT, x); }

/// Collection of vectors: `dim` CollOfScalar columns (equelleTypes.hpp:215-236).
class CollOfVector {
public:
    explicit CollOfVector(const int columns) : v(columns) {}
    const CollOfScalar& col(const int c) const { return v[c]; }
    CollOfScalar& col(const int c) { return v[c]; }
    const CollOfScalar& operator[](const int c) const { return v[c]; }
    CollOfScalar& operator[](const int c) { return v[c]; }
    int numCols() const { return (int)v.size(); }

private:
    std::vector<CollOfScalar> v;
};

inline CollOfVector operator+(const CollOfVector& v1, const CollOfVector& v2)
{
    CollOfVector res(v1.numCols());
    for (int d = 0; d < v1.numCols(); ++d) {
        res.col(d) = v1.col(d) + v2.col(d);
    }
    return res;
}
inline CollOfVector operator-(const CollOfVector& v1, const CollOfVector& v2)
{
    CollOfVector res(v1.numCols());
    for (int d = 0; d < v1.numCols(); ++d) {
        res.col(d) = v1.col(d) - v2.col(d);
    }
    return res;
}
inline CollOfVector operator-(const CollOfVector& x)
{
    CollOfVector res(x.numCols());
    for (int d = 0; d < x.numCols(); ++d) {
        res.col(d) = -x.col(d);
    }
    return res;
}
inline CollOfVector operator*(const CollOfVector& x, const Scalar& s)
{
    CollOfVector res(x.numCols());
    for (int d = 0; d < x.numCols(); ++d) {
        res.col(d) = x.col(d) * s;
    }
    return res;
}
inline CollOfVector operator*(const CollOfVector& x, const CollOfScalar& s)
{
    CollOfVector res(x.numCols());
    for (int d = 0; d < x.numCols(); ++d) {
        res.col(d) = x.col(d) * s;
    }
    return res;
}
inline CollOfVector operator*(const Scalar& s, const CollOfVector& x) { return x * s; }
inline CollOfVector operator*(const CollOfScalar& s, const CollOfVector& x) { return x * s; }
inline CollOfVector operator/(const CollOfVector& x, const Scalar& s)
{
    CollOfVector res(x.numCols());
    for (int d = 0; d < x.numCols(); ++d) {
        res.col(d) = x.col(d) / s;
    }
    return res;
}
inline CollOfVector operator/(const CollOfVector& x, const CollOfScalar& s)
{
    CollOfVector res(x.numCols());
    for (int d = 0; d < x.numCols(); ++d) {
        res.col(d) = x.col(d) / s;
    }
    return res;
}

/// Maps a collection type to the type a template result should have
/// (equelleTypes.hpp:321-324).
template <class Coll>
struct CollType {
    typedef Coll Type;
};

/// Array literals become tuples (equelleTypes.hpp:333-372).
template <typename T>
std::tuple<typename CollType<T>::Type> makeArray(const T& t)
{
    return std::tuple<typename CollType<T>::Type>{t};
}
template <typename T1, typename T2>
std::tuple<typename CollType<T1>::Type, typename CollType<T2>::Type> makeArray(const T1& t1, const T2& t2)
{
    return std::tuple<typename CollType<T1>::Type, typename CollType<T2>::Type>{t1, t2};
}
template <typename T1, typename T2, typename T3>
std::tuple<typename CollType<T1>::Type, typename CollType<T2>::Type, typename CollType<T3>::Type>
makeArray(const T1& t1, const T2& t2, const T3& t3)
{
    return std::tuple<typename CollType<T1>::Type, typename CollType<T2>::Type, typename CollType<T3>::Type>{
        t1, t2, t3};
}
template <typename T1, typename T2, typename T3, typename T4>
std::tuple<typename CollType<T1>::Type, typename CollType<T2>::Type, typename CollType<T3>::Type,
           typename CollType<T4>::Type>
makeArray(const T1& t1, const T2& t2, const T3& t3, const T4& t4)
{
    return std::tuple<typename CollType<T1>::Type, typename CollType<T2>::Type, typename CollType<T3>::Type,
                      typename CollType<T4>::Type>{t1, t2, t3, t4};
}

/// Residual function types for newtonSolveSystem (equelleTypes.hpp:374-400).
template <int Num>
struct ResCompType;
template <>
struct ResCompType<1> {
    typedef std::function<CollOfScalar(const CollOfScalar&)> type;
};
template <>
struct ResCompType<2> {
    typedef std::function<CollOfScalar(const CollOfScalar&, const CollOfScalar&)> type;
};
template <>
struct ResCompType<3> {
    typedef std::function<CollOfScalar(const CollOfScalar&, const CollOfScalar&, const CollOfScalar&)> type;
};
template <>
struct ResCompType<4> {
    typedef std::function<CollOfScalar(const CollOfScalar&, const CollOfScalar&, const CollOfScalar&,
                                       const CollOfScalar&)>
        type;
};

/// A strided index range (equelleTypes.hpp:407-498); newtonSolveSystem uses
/// unit-stride spans to split and recombine the unknowns.
class ESpan {
public:
    explicit ESpan(const int num) : num_(num), stride_(1), start_(0) {}
    ESpan(const int num, const int stride, const int start) : num_(num), stride_(stride), start_(start) {}
    int operator[](const int i) const
    {
        assert(i >= 0 && i < num_);
        return start_ + i * stride_;
    }
    int size() const { return num_; }
    int stride() const { return stride_; }
    int start() const { return start_; }
    bool operator==(const ESpan& rhs) const
    {
        return num_ == rhs.num_ && start_ == rhs.start_ && stride_ == rhs.stride_;
    }

private:
    int num_;
    int stride_;
    int start_;
};

}  // namespace equelle
