#pragma once
// Test infrastructure only (part of the oracle, never linked into the product library).
//
// A host-only stand-in for the small subset of the Kokkos 5.1 API that the reference's launch
// layer (src/exec) and solvers (src/solvers) use, so that those files compile unchanged and run
// on the CPU with Kokkos' Serial/OpenMP semantics: RangePolicy loops run on OpenMP threads,
// team policies run one member per team (team size 1, which is what the reference asks for on
// host backends: exec::simd_width() == 1), reductions and scans run serially. The reference's
// own kernels are written so that their results do not depend on the thread count
// (src/solvers/vector_ops.hpp:5-14, src/exec/force_settings.cpp:69-75), so OpenMP loops give the
// same bits as a serial run.
//
// Written for this project from the public Kokkos API; no Kokkos source is used.

#include <algorithm>
#include <cmath>
#include <cstddef>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <limits>
#include <memory>
#include <string>
#include <type_traits>
#include <utility>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

#define KOKKOS_INLINE_FUNCTION inline
#define KOKKOS_FORCEINLINE_FUNCTION inline
#define KOKKOS_FUNCTION
#define KOKKOS_LAMBDA [=]
#define KOKKOS_CLASS_LAMBDA [=, *this]
#define KOKKOS_VERSION 50100
#define KOKKOS_ENABLE_SERIAL 1

namespace Kokkos {

// ---------------------------------------------------------------- spaces, layouts, traits
struct ScratchMemorySpace {};
struct HostSpace {
  using memory_space = HostSpace;
};
struct Serial {
  using memory_space = HostSpace;
  using execution_space = Serial;
  using scratch_memory_space = ScratchMemorySpace;
  using size_type = std::size_t;
  static const char* name() { return "Serial"; }
  int concurrency() const {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
  }
  void fence(const std::string& = {}) const {}
};
using DefaultExecutionSpace = Serial;
using DefaultHostExecutionSpace = Serial;
using SharedHostPinnedSpace = HostSpace;

struct LayoutLeft {};
struct LayoutRight {};
enum MemoryTraitsFlags : unsigned { Unmanaged = 1u, RandomAccess = 2u, Atomic = 4u, Restrict = 8u };
template <unsigned N>
struct MemoryTraits {};
using MemoryUnmanaged = MemoryTraits<Unmanaged>;

struct ALL_t {};
inline constexpr ALL_t ALL{};

struct WithoutInitializing_t {};
inline constexpr WithoutInitializing_t WithoutInitializing{};

struct AllocProp {
  std::string label;
  bool initialize = true;
};
inline AllocProp view_alloc(WithoutInitializing_t, const std::string& label) { return {label, false}; }
inline AllocProp view_alloc(const std::string& label, WithoutInitializing_t) { return {label, false}; }
inline AllocProp view_alloc(const std::string& label) { return {label, true}; }

[[noreturn]] inline void abort(const char* msg) {
  std::fprintf(stderr, "Kokkos::abort: %s\n", msg);
  std::abort();
}
inline void fence(const std::string& = {}) {}

using std::floor;
using std::isfinite;
using std::sin;
using std::sqrt;
using std::abs;

template <class T>
inline void atomic_add(T* p, T v) {
#ifdef _OPENMP
#pragma omp atomic
#endif
  *p += v;
}

// ---------------------------------------------------------------- team scratch pool
// Each team member owns a bump allocator over a buffer sized by set_scratch_size.
struct ScratchPool {
  std::vector<unsigned char> buf;
  std::size_t used = 0;
  void* take(std::size_t bytes) {
    std::size_t off = (used + 15) / 16 * 16;
    if (off + bytes > buf.size()) Kokkos::abort("team scratch exhausted (shim)");
    used = off + bytes;
    return buf.data() + off;
  }
};

// ---------------------------------------------------------------- View
namespace detail {
template <class D>
struct Rank;
template <class T>
struct Rank {
  static constexpr int value = 0;
  using value_type = T;
};
template <class T>
struct Rank<T*> {
  static constexpr int value = 1 + Rank<T>::value;
  using value_type = typename Rank<T>::value_type;
};
template <class... P>
struct IsLayoutRight : std::false_type {};
template <class H, class... P>
struct IsLayoutRight<H, P...> : std::conditional_t<std::is_same_v<H, LayoutRight>, std::true_type, IsLayoutRight<P...>> {};
template <class... P>
struct IsLayoutLeft : std::false_type {};
template <class H, class... P>
struct IsLayoutLeft<H, P...> : std::conditional_t<std::is_same_v<H, LayoutLeft>, std::true_type, IsLayoutLeft<P...>> {};
}  // namespace detail

template <class DataType, class... Props>
class View {
 public:
  static constexpr int rank = detail::Rank<DataType>::value;
  using value_type = typename detail::Rank<DataType>::value_type;
  using non_const_value_type = std::remove_const_t<value_type>;
  using data_type = DataType;
  using memory_space = HostSpace;
  using execution_space = Serial;
  // Rank-2 views are LayoutLeft unless LayoutRight is named (the reference names LayoutLeft).
  static constexpr bool layout_right = detail::IsLayoutRight<Props...>::value;

  View() = default;

  View(const std::string& label, std::size_t n0 = 0, std::size_t n1 = 0) { allocate(label, n0, n1, true); }
  View(const char* label, std::size_t n0 = 0, std::size_t n1 = 0) { allocate(label, n0, n1, true); }
  View(const AllocProp& p, std::size_t n0 = 0, std::size_t n1 = 0) { allocate(p.label, n0, n1, p.initialize); }
  // Unmanaged wrap of existing memory.
  View(value_type* p, std::size_t n0 = 0, std::size_t n1 = 0) : ptr_(p) { set_extents(n0, n1); }
  // Team scratch.
  View(ScratchPool& pool, std::size_t n0 = 0, std::size_t n1 = 0) {
    set_extents(n0, n1);
    ptr_ = static_cast<value_type*>(pool.take(span() * sizeof(value_type)));
  }

  // Conversion (non-const -> const, or between property lists).
  template <class D2, class... P2,
            std::enable_if_t<std::is_convertible_v<typename View<D2, P2...>::value_type*, value_type*>, int> = 0>
  View(const View<D2, P2...>& o)
      : owner_(o.owner_), ptr_(o.ptr_), n0_(o.n0_), n1_(o.n1_), s0_(o.s0_), s1_(o.s1_), label_(o.label_) {}

  static std::size_t shmem_size(std::size_t n0 = 0, std::size_t n1 = 0) {
    return (rank >= 2 ? n0 * std::max<std::size_t>(n1, 1) : std::max<std::size_t>(n0, 1)) * sizeof(value_type) + 16;
  }

  value_type* data() const { return ptr_; }
  std::size_t extent(int r) const { return r == 0 ? (rank >= 1 ? n0_ : 1) : (rank >= 2 ? n1_ : 1); }
  int extent_int(int r) const { return static_cast<int>(extent(r)); }
  std::size_t size() const { return rank == 0 ? 1 : rank == 1 ? n0_ : n0_ * n1_; }
  std::size_t span() const { return size(); }
  std::size_t stride(int r) const { return r == 0 ? s0_ : s1_; }
  bool is_allocated() const { return ptr_ != nullptr; }
  const std::string& label() const { return label_; }
  bool span_is_contiguous() const { return rank <= 1 ? s0_ == 1 : (layout_right ? s1_ == 1 && s0_ == n1_ : s0_ == 1 && s1_ == n0_); }

  value_type& operator()() const { return ptr_[0]; }
  template <class I>
  value_type& operator()(I i) const {
    return ptr_[static_cast<std::ptrdiff_t>(i) * static_cast<std::ptrdiff_t>(s0_)];
  }
  template <class I, class J>
  value_type& operator()(I i, J j) const {
    return ptr_[static_cast<std::ptrdiff_t>(i) * static_cast<std::ptrdiff_t>(s0_) +
                static_cast<std::ptrdiff_t>(j) * static_cast<std::ptrdiff_t>(s1_)];
  }
  template <class I>
  value_type& operator[](I i) const {
    return (*this)(i);
  }

  // internals, public for subview/deep_copy
  std::shared_ptr<non_const_value_type> owner_;
  value_type* ptr_ = nullptr;
  std::size_t n0_ = 0, n1_ = 0, s0_ = 1, s1_ = 0;
  std::string label_;

  void set_extents(std::size_t n0, std::size_t n1) {
    n0_ = n0;
    n1_ = n1;
    if (rank >= 2) {
      if (layout_right) {
        s0_ = n1;
        s1_ = 1;
      } else {
        s0_ = 1;
        s1_ = n0;
      }
    } else {
      s0_ = 1;
      s1_ = 0;
    }
  }

 private:
  void allocate(const std::string& label, std::size_t n0, std::size_t n1, bool init) {
    label_ = label;
    set_extents(n0, n1);
    const std::size_t n = std::max<std::size_t>(span(), 1);
    owner_ = std::shared_ptr<non_const_value_type>(new non_const_value_type[n](),
                                                    std::default_delete<non_const_value_type[]>());
    (void)init;  // always value-initialized: a serial shim has nothing to gain from skipping it
    ptr_ = owner_.get();
  }
};

// ---------------------------------------------------------------- subview
template <class D, class... P>
View<typename View<D, P...>::value_type*, P...> subview(const View<D, P...>& v, std::pair<std::size_t, std::size_t> r) {
  static_assert(View<D, P...>::rank == 1);
  View<typename View<D, P...>::value_type*, P...> s;
  s.owner_ = v.owner_;
  s.ptr_ = v.ptr_ + static_cast<std::ptrdiff_t>(r.first * v.s0_);
  s.n0_ = r.second - r.first;
  s.s0_ = v.s0_;
  s.label_ = v.label_;
  return s;
}
template <class D, class... P, class A, class B>
View<typename View<D, P...>::value_type*, P...> subview(const View<D, P...>& v, std::pair<A, B> r) {
  return subview(v, std::pair<std::size_t, std::size_t>(static_cast<std::size_t>(r.first), static_cast<std::size_t>(r.second)));
}
template <class D, class... P, class I, std::enable_if_t<std::is_integral_v<I>, int> = 0>
View<typename View<D, P...>::value_type, P...> subview(const View<D, P...>& v, I i) {
  static_assert(View<D, P...>::rank == 1);
  View<typename View<D, P...>::value_type, P...> s;
  s.owner_ = v.owner_;
  s.ptr_ = v.ptr_ + static_cast<std::ptrdiff_t>(i) * static_cast<std::ptrdiff_t>(v.s0_);
  s.label_ = v.label_;
  return s;
}
// Column c of a rank-2 view.
template <class D, class... P, class I, std::enable_if_t<std::is_integral_v<I>, int> = 0>
View<typename View<D, P...>::value_type*, P...> subview(const View<D, P...>& v, ALL_t, I c) {
  View<typename View<D, P...>::value_type*, P...> s;
  s.owner_ = v.owner_;
  s.ptr_ = v.ptr_ + static_cast<std::ptrdiff_t>(c) * static_cast<std::ptrdiff_t>(v.s1_);
  s.n0_ = v.n0_;
  s.s0_ = v.s0_;
  s.label_ = v.label_;
  return s;
}
// Part of row i of a rank-2 view.
template <class D, class... P, class I, class A, class B, std::enable_if_t<std::is_integral_v<I>, int> = 0>
View<typename View<D, P...>::value_type*, P...> subview(const View<D, P...>& v, I i, std::pair<A, B> r) {
  View<typename View<D, P...>::value_type*, P...> s;
  s.owner_ = v.owner_;
  s.ptr_ = v.ptr_ + static_cast<std::ptrdiff_t>(i) * static_cast<std::ptrdiff_t>(v.s0_) +
           static_cast<std::ptrdiff_t>(r.first) * static_cast<std::ptrdiff_t>(v.s1_);
  s.n0_ = static_cast<std::size_t>(r.second - r.first);
  s.s0_ = v.s1_;
  s.label_ = v.label_;
  return s;
}

// ---------------------------------------------------------------- mirrors and copies
template <class D, class... P>
View<typename View<D, P...>::non_const_value_type*, P...> create_mirror_view(const View<D, P...>& v) {
  View<typename View<D, P...>::non_const_value_type*, P...> m;
  m.owner_ = std::const_pointer_cast<typename View<D, P...>::non_const_value_type>(v.owner_);
  m.ptr_ = const_cast<typename View<D, P...>::non_const_value_type*>(v.ptr_);
  m.n0_ = v.n0_;
  m.n1_ = v.n1_;
  m.s0_ = v.s0_;
  m.s1_ = v.s1_;
  m.label_ = v.label_;
  return m;
}
template <class S, class D, class... P>
auto create_mirror_view(const S&, const View<D, P...>& v) {
  return create_mirror_view(v);
}
template <class S, class D, class... P>
auto create_mirror_view_and_copy(const S&, const View<D, P...>& v) {
  return create_mirror_view(v);
}
template <class S, class D, class... P>
auto create_mirror(const S&, const View<D, P...>& v) {
  return create_mirror_view(v);
}

template <class D, class... P>
void deep_copy(const View<D, P...>& dst, const typename View<D, P...>::non_const_value_type& value) {
  using V = View<D, P...>;
  if constexpr (V::rank == 0) {
    *dst.ptr_ = value;
  } else if constexpr (V::rank == 1) {
    for (std::size_t i = 0; i < dst.n0_; ++i) dst(i) = value;
  } else {
    for (std::size_t j = 0; j < dst.n1_; ++j)
      for (std::size_t i = 0; i < dst.n0_; ++i) dst(i, j) = value;
  }
}
template <class D1, class... P1, class D2, class... P2>
void deep_copy(const View<D1, P1...>& dst, const View<D2, P2...>& src) {
  using V = View<D1, P1...>;
  if (static_cast<const void*>(dst.ptr_) == static_cast<const void*>(src.ptr_) && dst.s0_ == src.s0_ && dst.s1_ == src.s1_)
    return;
  if constexpr (V::rank == 0) {
    *dst.ptr_ = *src.ptr_;
  } else if constexpr (V::rank == 1) {
    if (dst.n0_ != src.n0_) Kokkos::abort("deep_copy: extents differ (shim)");
    for (std::size_t i = 0; i < dst.n0_; ++i) dst(i) = src(i);
  } else {
    if (dst.n0_ != src.n0_ || dst.n1_ != src.n1_) Kokkos::abort("deep_copy: extents differ (shim)");
    for (std::size_t j = 0; j < dst.n1_; ++j)
      for (std::size_t i = 0; i < dst.n0_; ++i) dst(i, j) = src(i, j);
  }
}
template <class T, class D, class... P, std::enable_if_t<std::is_arithmetic_v<T>, int> = 0>
void deep_copy(T& dst, const View<D, P...>& src) {
  dst = *src.ptr_;
}
template <class D1, class... P1, class D2, class... P2>
void deep_copy(const Serial&, const View<D1, P1...>& dst, const View<D2, P2...>& src) {
  deep_copy(dst, src);
}

// ---------------------------------------------------------------- policies
template <class T>
struct IndexType {};

template <class... Args>
struct RangePolicy {
  std::int64_t begin = 0, end = 0;
  RangePolicy() = default;
  template <class A, class B>
  RangePolicy(A b, B e) : begin(static_cast<std::int64_t>(b)), end(static_cast<std::int64_t>(e)) {}
  template <class S, class A, class B, std::enable_if_t<!std::is_integral_v<S>, int> = 0>
  RangePolicy(const S&, A b, B e) : begin(static_cast<std::int64_t>(b)), end(static_cast<std::int64_t>(e)) {}
};

struct AUTO_t {};
inline constexpr AUTO_t AUTO{};
struct ParallelForTag {};

struct ScratchRequest {
  std::size_t bytes = 0;
  bool per_thread = false;
};
inline ScratchRequest PerTeam(std::size_t b) { return {b, false}; }
inline ScratchRequest PerThread(std::size_t b) { return {b, true}; }

class TeamMember {
 public:
  TeamMember(int league_rank, int league_size, ScratchPool* team, ScratchPool* thread)
      : league_rank_(league_rank), league_size_(league_size), team_(team), thread_(thread) {}
  int league_rank() const { return league_rank_; }
  int league_size() const { return league_size_; }
  int team_rank() const { return 0; }
  int team_size() const { return 1; }
  ScratchPool& team_scratch(int) const { return *team_; }
  ScratchPool& thread_scratch(int) const { return *thread_; }
  void team_barrier() const {}

 private:
  int league_rank_, league_size_;
  ScratchPool *team_, *thread_;
};

struct SingleTeam {
  const TeamMember* m;
};
struct SingleThread {
  const TeamMember* m;
};
inline SingleTeam PerTeam(const TeamMember& m) { return {&m}; }
inline SingleThread PerThread(const TeamMember& m) { return {&m}; }
template <class F>
void single(const SingleTeam&, F&& f) {
  f();
}
template <class F>
void single(const SingleThread&, F&& f) {
  f();
}
template <class F, class T>
void single(const SingleTeam&, F&& f, T& v) {
  f(v);
}

template <class... Args>
class TeamPolicy {
 public:
  using member_type = TeamMember;
  TeamPolicy() = default;
  TeamPolicy(int league, int team, int = 1) : league_(league), team_(team) {}
  TeamPolicy(int league, AUTO_t, int = 1) : league_(league), team_(1) {}
  template <class S, std::enable_if_t<!std::is_integral_v<S>, int> = 0>
  TeamPolicy(const S&, int league, int team, int = 1) : league_(league), team_(team) {}
  TeamPolicy& set_scratch_size(int, ScratchRequest a) {
    (a.per_thread ? thread_bytes_ : team_bytes_) += a.bytes;
    return *this;
  }
  TeamPolicy& set_scratch_size(int, ScratchRequest a, ScratchRequest b) {
    set_scratch_size(0, a);
    return set_scratch_size(0, b);
  }
  template <class F, class Tag>
  int team_size_max(const F&, Tag) const {
    return 1;
  }
  template <class F, class Tag>
  int team_size_recommended(const F&, Tag) const {
    return 1;
  }
  static std::size_t scratch_size_max(int) { return std::size_t(1) << 30; }
  int league_size() const { return league_; }
  int team_size() const { return team_; }
  std::size_t team_bytes_ = 0, thread_bytes_ = 0;

 private:
  int league_ = 0, team_ = 1;
};

struct TeamThreadRangeBoundaries {
  std::int64_t begin, end;
};
template <class I>
TeamThreadRangeBoundaries TeamThreadRange(const TeamMember&, I n) {
  return {0, static_cast<std::int64_t>(n)};
}
template <class I, class J>
TeamThreadRangeBoundaries TeamThreadRange(const TeamMember&, I b, J e) {
  return {static_cast<std::int64_t>(b), static_cast<std::int64_t>(e)};
}
struct ThreadVectorRangeBoundaries {
  std::int64_t begin, end;
};
template <class I>
ThreadVectorRangeBoundaries ThreadVectorRange(const TeamMember&, I n) {
  return {0, static_cast<std::int64_t>(n)};
}
template <class I, class J>
ThreadVectorRangeBoundaries ThreadVectorRange(const TeamMember&, I b, J e) {
  return {static_cast<std::int64_t>(b), static_cast<std::int64_t>(e)};
}

// ---------------------------------------------------------------- dispatch
namespace detail {
template <class F>
void range_for(std::int64_t b, std::int64_t e, const F& f) {
#ifdef _OPENMP
#pragma omp parallel for schedule(static)
#endif
  for (std::int64_t i = b; i < e; ++i) f(i);
}
}  // namespace detail

template <class... A, class F>
void parallel_for(const std::string&, const RangePolicy<A...>& p, const F& f) {
  detail::range_for(p.begin, p.end, [&](std::int64_t i) { f(i); });
}
template <class... A, class F>
void parallel_for(const RangePolicy<A...>& p, const F& f) {
  parallel_for(std::string(), p, f);
}
template <class I, class F, std::enable_if_t<std::is_integral_v<I>, int> = 0>
void parallel_for(const std::string&, I n, const F& f) {
  detail::range_for(0, static_cast<std::int64_t>(n), [&](std::int64_t i) { f(i); });
}
template <class... A, class F>
void parallel_for(const std::string&, const TeamPolicy<A...>& p, const F& f) {
  if (p.team_size() != 1) Kokkos::abort("team policies with more than one member are not supported by the shim");
  const int league = p.league_size();
#ifdef _OPENMP
#pragma omp parallel
#endif
  {
    ScratchPool team, thread;
    team.buf.resize(p.team_bytes_ + 64);
    thread.buf.resize(p.thread_bytes_ + 64);
#ifdef _OPENMP
#pragma omp for schedule(static)
#endif
    for (int r = 0; r < league; ++r) {
      team.used = 0;
      thread.used = 0;
      TeamMember m(r, league, &team, &thread);
      f(m);
    }
  }
}
template <class F>
void parallel_for(const TeamThreadRangeBoundaries& r, const F& f) {
  for (std::int64_t i = r.begin; i < r.end; ++i) f(static_cast<int>(i));
}
template <class F>
void parallel_for(const ThreadVectorRangeBoundaries& r, const F& f) {
  for (std::int64_t i = r.begin; i < r.end; ++i) f(static_cast<int>(i));
}

template <class T>
struct Min {
  T& ref;
  explicit Min(T& r) : ref(r) {}
  using value_type = T;
};
template <class T>
struct Max {
  T& ref;
  explicit Max(T& r) : ref(r) {}
  using value_type = T;
};
template <class T>
struct Sum {
  T& ref;
  explicit Sum(T& r) : ref(r) {}
  using value_type = T;
};

template <class... A, class F, class T>
void parallel_reduce(const std::string&, const RangePolicy<A...>& p, const F& f, Min<T> m) {
  T v = std::numeric_limits<T>::max();
  for (std::int64_t i = p.begin; i < p.end; ++i) f(i, v);
  m.ref = v;
}
template <class... A, class F, class T>
void parallel_reduce(const std::string&, const RangePolicy<A...>& p, const F& f, Max<T> m) {
  T v = std::numeric_limits<T>::lowest();
  for (std::int64_t i = p.begin; i < p.end; ++i) f(i, v);
  m.ref = v;
}
template <class... A, class F, class T>
void parallel_reduce(const std::string&, const RangePolicy<A...>& p, const F& f, Sum<T> s) {
  T v = T();
  for (std::int64_t i = p.begin; i < p.end; ++i) f(i, v);
  s.ref = v;
}
template <class... A, class F, class T, std::enable_if_t<std::is_arithmetic_v<T>, int> = 0>
void parallel_reduce(const std::string&, const RangePolicy<A...>& p, const F& f, T& result) {
  T v = T();
  for (std::int64_t i = p.begin; i < p.end; ++i) f(i, v);
  result = v;
}

template <class... A, class F, class T>
void parallel_scan(const std::string&, const RangePolicy<A...>& p, const F& f, T& total) {
  T v = T();
  for (std::int64_t i = p.begin; i < p.end; ++i) f(static_cast<T>(i), v, true);
  total = v;
}
template <class... A, class F>
void parallel_scan(const std::string& l, const RangePolicy<A...>& p, const F& f) {
  std::int64_t t = 0;
  std::int64_t v = 0;
  for (std::int64_t i = p.begin; i < p.end; ++i) f(i, v, true);
  (void)t;
  (void)l;
}

// ---------------------------------------------------------------- runtime
class ScopeGuard {
 public:
  ScopeGuard(int&, char**) {}
  ScopeGuard() = default;
};
inline void initialize(int&, char**) {}
inline void finalize() {}
inline bool is_initialized() { return true; }

}  // namespace Kokkos
