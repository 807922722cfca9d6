// Kokkos-subset shim (test infrastructure only).
//
// Lets the reference sources compile unmodified on the host so that the
// real reference can be run here as the CPU checker and CPU baseline. It
// covers exactly the Kokkos API the reference uses (`grep -oh "Kokkos::[A-Za-z_]*"
// src/*`): rank-1..8 LayoutRight Views with shared ownership and
// zero-initialised storage, resize, deep_copy, create_mirror_view(_and_copy),
// RangePolicy<IndexType<unsigned>>, parallel_for, parallel_reduce with
// Min<double> or a plain double sum, fence, Timer, initialize/finalize.
// parallel_for/parallel_reduce run over OpenMP when compiled with -fopenmp.
// Every flat index writes distinct memory in the reference kernels and the
// min-reduction is order independent, so results do not depend on the
// thread count.
#pragma once
#include <algorithm>
#include <cassert>
#include <chrono>
#include <cmath>
#include <cstddef>
#include <cstdint>
#include <cstring>
#include <limits>
#include <memory>
#include <string>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

#define KOKKOS_INLINE_FUNCTION inline
#define KOKKOS_LAMBDA [=]

namespace Kokkos {

struct LayoutRight {};
struct HostSpace { using execution_space = HostSpace; };
struct CudaSpace { using execution_space = CudaSpace; };
struct CudaUVMSpace { using execution_space = CudaUVMSpace; };

namespace impl {
template <class T> struct rank_of { static constexpr int value = 0; using scalar = T; };
template <class T> struct rank_of<T*> {
    static constexpr int value = 1 + rank_of<T>::value;
    using scalar = typename rank_of<T>::scalar;
};
}  // namespace impl

template <class DataType, class... Props>
class View {
  public:
    static constexpr int Rank = impl::rank_of<DataType>::value;
    using value_type = typename impl::rank_of<DataType>::scalar;
    using host_mirror_type = View<DataType, Props...>;

    View() { std::fill(ext_, ext_ + 8, 0); }
    explicit View(const std::string&) : View() {}
    template <class... N>
    View(const std::string&, N... n) : View() {
        static_assert(sizeof...(N) == Rank, "wrong number of extents");
        const size_t dims[] = {size_t(n)...};
        allocate(dims);
    }

    void allocate(const size_t* n) {
        size_t total = 1;
        for (int r = 0; r < Rank; r++) { ext_[r] = n[r]; total *= n[r]; }
        for (int r = Rank; r < 8; r++) ext_[r] = 1;
        store_ = std::make_shared<std::vector<value_type>>(total, value_type(0));
        ptr_ = store_->data();
        size_ = total;
        size_t s = 1;
        for (int r = Rank - 1; r >= 0; r--) { stride_[r] = s; s *= ext_[r]; }
    }

    value_type* data() const { return ptr_; }
    size_t size() const { return size_; }
    size_t span() const { return size_; }
    size_t extent(int r) const { return ext_[r]; }

    template <class... Idx>
    value_type& operator()(Idx... idx) const {
        static_assert(sizeof...(Idx) == Rank, "wrong number of indices");
        const size_t ids[] = {size_t(idx)...};
        size_t off = 0;
        for (int r = 0; r < Rank; r++) off += ids[r] * stride_[r];
        return ptr_[off];
    }
    value_type& operator[](size_t i) const { return ptr_[i * stride_[0]]; }

  private:
    std::shared_ptr<std::vector<value_type>> store_;
    value_type* ptr_ = nullptr;
    size_t size_ = 0;
    size_t ext_[8];
    size_t stride_[8] = {0, 0, 0, 0, 0, 0, 0, 0};
};

// Kokkos::resize keeps the overlapping contents; the reference only resizes
// views that are empty or have the same shape, so copying the overlap of
// the flat storage is sufficient for it.
template <class V, class... N>
void resize(V& v, N... n) {
    const size_t dims[] = {size_t(n)...};
    static_assert(sizeof...(N) == V::Rank, "wrong number of extents");
    V nv;
    nv.allocate(dims);
    if (v.data() && v.size() == nv.size())
        std::memcpy(nv.data(), v.data(), v.size() * sizeof(typename V::value_type));
    v = nv;
}

template <class V>
void deep_copy(const V& dst, const typename V::value_type& val) {
    std::fill(dst.data(), dst.data() + dst.size(), val);
}
template <class V, class... P>
void deep_copy(const V& dst, const View<P...>& src) {
    assert(dst.size() == src.size());
    if (dst.data() != src.data())
        std::memcpy(dst.data(), src.data(), dst.size() * sizeof(typename V::value_type));
}

template <class V> V create_mirror_view(const V& v) { return v; }
template <class S, class V> V create_mirror_view_and_copy(const S&, const V& v) { return v; }

template <class T> struct IndexType { using type = T; };

template <class... Args>
struct RangePolicy {
    unsigned begin, end;
    RangePolicy(unsigned b, unsigned e) : begin(b), end(e) {}
};

template <class T>
struct Min {
    T& ref;
    explicit Min(T& r) : ref(r) {}
};

template <class Policy, class F>
void parallel_for(const char*, const Policy& p, const F& f) {
    const long b = p.begin, e = p.end;
#pragma omp parallel for schedule(static)
    for (long i = b; i < e; i++) f(unsigned(i));
}
template <class Policy, class F>
void parallel_for(const std::string& l, const Policy& p, const F& f) { parallel_for(l.c_str(), p, f); }

template <class Policy, class F>
void parallel_reduce(const char*, const Policy& p, const F& f, Min<double> m) {
    const long b = p.begin, e = p.end;
    double result = std::numeric_limits<double>::max();
#pragma omp parallel
    {
        double local = std::numeric_limits<double>::max();
#pragma omp for schedule(static)
        for (long i = b; i < e; i++) f(unsigned(i), local);
#pragma omp critical
        result = result < local ? result : local;
    }
    m.ref = result;
}

template <class Policy, class F>
void parallel_reduce(const char*, const Policy& p, const F& f, double& sum) {
    // Serial on purpose: a fixed summation order keeps diagnostics reproducible.
    double s = 0;
    for (long i = p.begin; i < long(p.end); i++) f(unsigned(i), s);
    sum = s;
}

inline void fence() {}
inline void initialize(int&, char**) {}
inline void finalize() {}

class Timer {
  public:
    Timer() : t0_(std::chrono::steady_clock::now()) {}
    double seconds() const {
        return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0_).count();
    }
    void reset() { t0_ = std::chrono::steady_clock::now(); }

  private:
    std::chrono::steady_clock::time_point t0_;
};

}  // namespace Kokkos
