// oracle/kokkos_compat/Kokkos_Core.hpp
//
// TEST INFRASTRUCTURE ONLY. A host-only stand-in for the subset of Kokkos 5.2 that the
// reference's hot-path C++ (ww3-gpu kokkos/src/ww_kokkos/snl1_*, its fortran_iface shims)
// uses, so that those files compile unmodified with g++ into the CPU oracle under
// oracle/_ref/. Nothing in the product library includes this header.
//
// Semantics kept from Kokkos where the reference depends on them:
//   * A team is one host thread (team_size 1). TeamThreadRange covers the whole range in
//     order, so a team_barrier between two ranges is a no-op, and a kernel with no
//     reduction (W3SNL1, kokkos/src/ww_kokkos/snl1_team.hpp:18-20) computes the same bits
//     as on any Kokkos backend.
//   * The league of a TeamPolicy runs over OpenMP threads, schedule(dynamic, chunk), the
//     way Kokkos' OpenMP backend runs it; each thread owns a team-scratch bump buffer.
//   * View is a reference-counted handle; LayoutLeft is column-major, LayoutRight (the
//     host default) row-major; an unmanaged View wraps a caller's pointer.
//   * Kokkos::max(a, b) is (a < b) ? b : a and Kokkos::min(a, b) is (b < a) ? b : a.
//   * Math functions forward to the C library's float or double overloads (glibc on this
//     host), which is what Kokkos' host math does.
#pragma once

#include <omp.h>

#include <algorithm>
#include <array>
#include <cmath>
#include <cstddef>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <cstdio>
#include <cstdlib>
#include <functional>
#include <limits>
#include <memory>
#include <string>
#include <type_traits>
#include <utility>
#include <vector>

#define KOKKOS_ENABLE_OPENMP 1
#define KOKKOS_ENABLE_SERIAL 1
#define KOKKOS_LAMBDA [=]
#define KOKKOS_CLASS_LAMBDA [ =, *this ]
#define KOKKOS_FUNCTION
#define KOKKOS_INLINE_FUNCTION inline
#define KOKKOS_FORCEINLINE_FUNCTION inline __attribute__((always_inline))
#define KOKKOS_DEFAULTED_FUNCTION
#define KOKKOS_IMPL_COMPAT_STRIP(...) __VA_ARGS__
#define KOKKOS_IF_ON_HOST(CODE) { KOKKOS_IMPL_COMPAT_STRIP CODE }
#define KOKKOS_IF_ON_DEVICE(CODE) {}
#define KOKKOS_ASSERT(x) ((void)0)

namespace Kokkos {

// ---------------------------------------------------------------- memory and layouts
struct LayoutLeft {};
struct LayoutRight {};
struct LayoutStride {};
struct HostSpace {
  using memory_space = HostSpace;
  static constexpr const char* name() { return "HostSpace"; }
};
enum MemoryTraitsFlags : unsigned { Unmanaged = 0x01, RandomAccess = 0x02, Atomic = 0x04, Restrict = 0x08 };
template <unsigned Flags>
struct MemoryTraits {
  static constexpr unsigned value = Flags;
};

struct WithoutInitializing_t {};
inline constexpr WithoutInitializing_t WithoutInitializing{};
struct ALL_t {};
inline constexpr ALL_t ALL{};

template <class A, class B>
using pair = std::pair<A, B>;
template <class A, class B>
constexpr std::pair<A, B> make_pair(A a, B b) { return std::pair<A, B>(a, b); }

/// Bump allocator behind team_scratch(level): one per executing host thread.
class ScratchMemorySpace {
 public:
  ScratchMemorySpace() = default;
  ScratchMemorySpace(char* base, std::size_t size) : base_(base), size_(size), used_(0) {}
  void* get_shmem(std::size_t bytes) {
    const std::size_t align = 8;
    used_ = (used_ + align - 1) / align * align;
    if (used_ + bytes > size_) std::abort();  // a request beyond set_scratch_size
    void* p = base_ + used_;
    used_ += bytes;
    return p;
  }
  using memory_space = ScratchMemorySpace;
  using execution_space = void;

 private:
  char* base_ = nullptr;
  std::size_t size_ = 0;
  std::size_t used_ = 0;
};

namespace Impl {
template <class T>
struct view_rank { static constexpr int value = 0; using value_type = T; };
template <class T>
struct view_rank<T*> {
  static constexpr int value = 1 + view_rank<T>::value;
  using value_type = typename view_rank<T>::value_type;
};
template <class T, std::size_t N>
struct view_rank<T[N]> {
  static constexpr int value = 1 + view_rank<T>::value;
  using value_type = typename view_rank<T>::value_type;
};

template <class... P>
struct view_props {
  using layout = LayoutRight;
  static constexpr bool unmanaged = false;
};
template <class... P>
struct view_props<LayoutLeft, P...> : view_props<P...> { using layout = LayoutLeft; };
template <class... P>
struct view_props<LayoutRight, P...> : view_props<P...> { using layout = LayoutRight; };
template <unsigned F, class... P>
struct view_props<MemoryTraits<F>, P...> : view_props<P...> {
  static constexpr bool unmanaged = (F & Unmanaged) != 0 || view_props<P...>::unmanaged;
};
template <class Other, class... P>
struct view_props<Other, P...> : view_props<P...> {};

struct AllocProp {
  std::string label;
  bool init = true;
};
inline void fill_prop(AllocProp&) {}
template <class... R>
void fill_prop(AllocProp& p, const std::string& s, const R&... r) { p.label = s; fill_prop(p, r...); }
template <class... R>
void fill_prop(AllocProp& p, const char* s, const R&... r) { p.label = s; fill_prop(p, r...); }
template <class... R>
void fill_prop(AllocProp& p, WithoutInitializing_t, const R&... r) { p.init = false; fill_prop(p, r...); }
template <class X, class... R>
void fill_prop(AllocProp& p, const X&, const R&... r) { fill_prop(p, r...); }  // execution spaces
}  // namespace Impl

template <class... Args>
Impl::AllocProp view_alloc(const Args&... args) {
  Impl::AllocProp p;
  Impl::fill_prop(p, args...);
  return p;
}

template <class DataType, class... Props>
class View {
 public:
  static constexpr int Rank = Impl::view_rank<DataType>::value;
  static constexpr std::integral_constant<int, Rank> rank{};  // callable, as in Kokkos 4
  using value_type = typename Impl::view_rank<DataType>::value_type;
  using non_const_value_type = std::remove_const_t<value_type>;
  using const_value_type = std::add_const_t<value_type>;
  using pointer_type = value_type*;
  using reference_type = value_type&;
  using array_layout = typename Impl::view_props<Props...>::layout;
  using memory_space = HostSpace;
  using device_type = HostSpace;
  using execution_space = void;
  using HostMirror = View;
  using host_mirror_type = View;
  using data_type = DataType;
  static constexpr bool kUnmanaged = Impl::view_props<Props...>::unmanaged;

  View() = default;

  // Managed allocation, zero-filled unless WithoutInitializing.
  View(const std::string& label, std::size_t n0 = 0, std::size_t n1 = 0, std::size_t n2 = 0,
       std::size_t n3 = 0) {
    allocate(label, true, n0, n1, n2, n3);
  }
  View(const char* label, std::size_t n0 = 0, std::size_t n1 = 0, std::size_t n2 = 0,
       std::size_t n3 = 0) {
    allocate(label, true, n0, n1, n2, n3);
  }
  View(const Impl::AllocProp& p, std::size_t n0 = 0, std::size_t n1 = 0, std::size_t n2 = 0,
       std::size_t n3 = 0) {
    allocate(p.label, p.init, n0, n1, n2, n3);
  }
  // Wrap a caller's pointer (unmanaged, whatever the traits say).
  View(pointer_type ptr, std::size_t n0 = 0, std::size_t n1 = 0, std::size_t n2 = 0,
       std::size_t n3 = 0) {
    ptr_ = ptr;
    set_extents(n0, n1, n2, n3);
  }
  // Team or thread scratch.
  View(ScratchMemorySpace& space, std::size_t n0 = 0, std::size_t n1 = 0, std::size_t n2 = 0,
       std::size_t n3 = 0) {
    set_extents(n0, n1, n2, n3);
    ptr_ = static_cast<pointer_type>(space.get_shmem(span() * sizeof(value_type)));
  }
  // Conversion from a View with a compatible (non-const -> const) value type and layout.
  template <class D2, class... P2,
            class = std::enable_if_t<
                View<D2, P2...>::Rank == Rank &&
                (Rank <= 1 ||
                 std::is_same_v<typename View<D2, P2...>::array_layout, array_layout>) &&
                std::is_convertible_v<typename View<D2, P2...>::value_type*, value_type*>>>
  View(const View<D2, P2...>& o) {
    ptr_ = o.data();
    owner_ = o.impl_owner();
    for (int r = 0; r < 4; ++r) ext_[r] = o.extent(r);
    label_ = o.label();
  }

  static std::size_t shmem_size(std::size_t n0 = 0, std::size_t n1 = 0, std::size_t n2 = 0,
                                std::size_t n3 = 0) {
    const std::size_t n[4] = {n0, n1, n2, n3};
    std::size_t s = 1;
    for (int r = 0; r < Rank; ++r) s *= n[r];
    return s * sizeof(value_type) + 8;  // + alignment slack of the bump allocator
  }

  pointer_type data() const { return ptr_; }
  std::size_t extent(int r) const { return r < 4 ? ext_[r] : 1; }
  int extent_int(int r) const { return static_cast<int>(extent(r)); }
  std::size_t size() const { return span(); }
  std::size_t span() const {
    std::size_t s = 1;
    for (int r = 0; r < Rank; ++r) s *= ext_[r];
    return Rank == 0 ? 1 : s;
  }
  bool span_is_contiguous() const { return true; }
  bool is_allocated() const { return ptr_ != nullptr; }
  const std::string& label() const { return label_; }
  std::size_t stride(int r) const {
    std::size_t s = 1;
    if constexpr (std::is_same_v<array_layout, LayoutLeft>) {
      for (int q = 0; q < r; ++q) s *= ext_[q];
    } else {
      for (int q = Rank - 1; q > r; --q) s *= ext_[q];
    }
    return s;
  }
  std::size_t stride_0() const { return stride(0); }
  std::size_t stride_1() const { return stride(1); }
  const std::shared_ptr<void>& impl_owner() const { return owner_; }

  reference_type operator()() const { return ptr_[0]; }
  template <class I0>
  reference_type operator()(I0 i0) const { return ptr_[static_cast<std::ptrdiff_t>(i0)]; }
  template <class I0, class I1>
  reference_type operator()(I0 i0, I1 i1) const {
    return ptr_[offset(static_cast<std::size_t>(i0), static_cast<std::size_t>(i1), 0, 0)];
  }
  template <class I0, class I1, class I2>
  reference_type operator()(I0 i0, I1 i1, I2 i2) const {
    return ptr_[offset(static_cast<std::size_t>(i0), static_cast<std::size_t>(i1),
                       static_cast<std::size_t>(i2), 0)];
  }
  template <class I0, class I1, class I2, class I3>
  reference_type operator()(I0 i0, I1 i1, I2 i2, I3 i3) const {
    return ptr_[offset(static_cast<std::size_t>(i0), static_cast<std::size_t>(i1),
                       static_cast<std::size_t>(i2), static_cast<std::size_t>(i3))];
  }
  template <class I0>
  reference_type operator[](I0 i0) const { return ptr_[static_cast<std::ptrdiff_t>(i0)]; }

  // Internal: a view of the same memory with new extents (subview).
  static View impl_wrap(pointer_type p, const std::shared_ptr<void>& owner, std::size_t n0,
                        std::size_t n1 = 0, std::size_t n2 = 0, std::size_t n3 = 0) {
    View v;
    v.ptr_ = p;
    v.owner_ = owner;
    v.set_extents(n0, n1, n2, n3);
    return v;
  }

 private:
  void set_extents(std::size_t n0, std::size_t n1, std::size_t n2, std::size_t n3) {
    const std::size_t n[4] = {n0, n1, n2, n3};
    for (int r = 0; r < 4; ++r) ext_[r] = r < Rank ? n[r] : 1;
  }
  void allocate(const std::string& label, bool init, std::size_t n0, std::size_t n1,
                std::size_t n2, std::size_t n3) {
    label_ = label;
    set_extents(n0, n1, n2, n3);
    const std::size_t n = span();
    auto* raw = static_cast<non_const_value_type*>(std::malloc((n ? n : 1) * sizeof(value_type)));
    if (raw == nullptr) throw std::bad_alloc();
    if (init) std::memset(static_cast<void*>(raw), 0, n * sizeof(value_type));
    owner_ = std::shared_ptr<void>(static_cast<void*>(raw), [](void* q) { std::free(q); });
    ptr_ = raw;
  }
  std::size_t offset(std::size_t i0, std::size_t i1, std::size_t i2, std::size_t i3) const {
    if constexpr (std::is_same_v<array_layout, LayoutLeft>) {
      return i0 + ext_[0] * (i1 + ext_[1] * (i2 + ext_[2] * i3));
    } else {
      if constexpr (Rank == 2) return i0 * ext_[1] + i1;
      if constexpr (Rank == 3) return (i0 * ext_[1] + i1) * ext_[2] + i2;
      return ((i0 * ext_[1] + i1) * ext_[2] + i2) * ext_[3] + i3;
    }
  }

  pointer_type ptr_ = nullptr;
  std::shared_ptr<void> owner_;
  std::size_t ext_[4] = {0, 0, 0, 0};
  std::string label_;
};

// ---------------------------------------------------------------- subviews
template <class D, class... P>
View<D, P...> subview(const View<D, P...>& v, std::pair<int, int> r) {
  return View<D, P...>::impl_wrap(v.data() + r.first, v.impl_owner(),
                                  static_cast<std::size_t>(r.second - r.first));
}
template <class D, class... P>
View<D, P...> subview(const View<D, P...>& v, ALL_t, std::pair<int, int> r) {
  static_assert(std::is_same_v<typename View<D, P...>::array_layout, LayoutLeft>,
                "column ranges of a LayoutLeft view only");
  return View<D, P...>::impl_wrap(v.data() + v.extent(0) * static_cast<std::size_t>(r.first),
                                  v.impl_owner(), v.extent(0),
                                  static_cast<std::size_t>(r.second - r.first));
}
template <class D, class... P>
auto subview(const View<D, P...>& v, ALL_t, int col) {
  using V1 = View<typename View<D, P...>::value_type*, LayoutLeft, HostSpace>;
  return V1::impl_wrap(v.data() + v.extent(0) * static_cast<std::size_t>(col), v.impl_owner(),
                       v.extent(0));
}

// ---------------------------------------------------------------- copies and mirrors
template <class D1, class... P1, class D2, class... P2>
void deep_copy(const View<D1, P1...>& dst, const View<D2, P2...>& src) {
  if (static_cast<const void*>(dst.data()) == static_cast<const void*>(src.data())) return;
  const std::size_t n = std::min(dst.span(), src.span());
  std::memmove(static_cast<void*>(dst.data()), static_cast<const void*>(src.data()),
               n * sizeof(typename View<D1, P1...>::value_type));
}
template <class Exec, class D1, class... P1, class D2, class... P2>
void deep_copy(const Exec&, const View<D1, P1...>& dst, const View<D2, P2...>& src) {
  deep_copy(dst, src);
}
template <class D1, class... P1>
void deep_copy(const View<D1, P1...>& dst, const typename View<D1, P1...>::const_value_type& value) {
  for (std::size_t i = 0; i < dst.span(); ++i) dst.data()[i] = value;
}
template <class Exec, class D1, class... P1>
void deep_copy(const Exec&, const View<D1, P1...>& dst,
               const typename View<D1, P1...>::const_value_type& value) {
  deep_copy(dst, value);
}
template <class D, class... P>
View<D, P...> create_mirror_view(const View<D, P...>& v) { return v; }
template <class S, class D, class... P>
View<D, P...> create_mirror_view(const S&, const View<D, P...>& v) { return v; }
template <class S, class D, class... P>
View<D, P...> create_mirror_view_and_copy(const S&, const View<D, P...>& v) { return v; }
template <class D, class... P>
auto create_mirror(const View<D, P...>& v) {
  using V = View<typename View<D, P...>::non_const_value_type*, P...>;
  View<D, P...> m(std::string(v.label()) + "_mirror", v.extent(0), v.extent(1), v.extent(2),
                  v.extent(3));
  deep_copy(m, v);
  return m;
}

// ---------------------------------------------------------------- execution spaces
namespace Impl {
inline bool& initialized_flag() { static bool f = false; return f; }
inline bool& finalized_flag() { static bool f = false; return f; }
inline std::vector<std::function<void()>>& finalize_hooks() {
  static auto* v = new std::vector<std::function<void()>>();
  return *v;
}
}  // namespace Impl

class OpenMP {
 public:
  using execution_space = OpenMP;
  using memory_space = HostSpace;
  using scratch_memory_space = ScratchMemorySpace;
  using size_type = std::size_t;
  static int concurrency() { return omp_get_max_threads(); }
  int concurrency_instance() const { return omp_get_max_threads(); }
  void fence(const std::string& = "") const {}
  static void impl_static_fence(const std::string& = "") {}
  static constexpr const char* name() { return "OpenMP"; }
  static constexpr bool kParallel = true;
};
class Serial {
 public:
  using execution_space = Serial;
  using memory_space = HostSpace;
  using scratch_memory_space = ScratchMemorySpace;
  using size_type = std::size_t;
  static int concurrency() { return 1; }
  void fence(const std::string& = "") const {}
  static constexpr const char* name() { return "Serial"; }
  static constexpr bool kParallel = false;
};
using DefaultExecutionSpace = OpenMP;
using DefaultHostExecutionSpace = OpenMP;

template <class Space, class MemSpace>
struct SpaceAccessibility {
  static constexpr bool accessible = true;
  static constexpr bool assignable = true;
};

struct InitializationSettings {
  InitializationSettings& set_device_id(int) { return *this; }
  InitializationSettings& set_num_threads(int) { return *this; }
  InitializationSettings& set_disable_warnings(bool) { return *this; }
};
inline void initialize(const InitializationSettings& = {}) {
  Impl::initialized_flag() = true;
  Impl::finalized_flag() = false;
}
inline void initialize(int&, char**) { initialize(); }
inline bool is_initialized() { return Impl::initialized_flag(); }

/// Kokkos::abort: print the message and stop, as Kokkos does on the host.
[[noreturn]] inline void abort(const char* msg) {
  std::fprintf(stderr, "Kokkos::abort: %s\n", msg);
  std::abort();
}
inline bool is_finalized() { return Impl::finalized_flag(); }
inline void push_finalize_hook(std::function<void()> f) {
  Impl::finalize_hooks().push_back(std::move(f));
}
inline void finalize() {
  auto& hooks = Impl::finalize_hooks();
  for (auto it = hooks.rbegin(); it != hooks.rend(); ++it) (*it)();
  hooks.clear();
  Impl::initialized_flag() = false;
  Impl::finalized_flag() = true;
}
inline void fence(const std::string& = "") {}

namespace Profiling {
inline void pushRegion(const std::string&) {}
inline void popRegion() {}
}  // namespace Profiling

// ---------------------------------------------------------------- policies
struct AUTO_t {};
inline constexpr AUTO_t AUTO{};
struct Dynamic {};
struct Static {};
template <class T>
struct Schedule { using type = T; };
template <class T>
struct IndexType { using type = T; };

struct ParallelForTag {};
struct ParallelReduceTag {};

struct PerTeamValue { std::size_t value; };
struct PerThreadValue { std::size_t value; };
inline PerTeamValue PerTeam(std::size_t v) { return PerTeamValue{v}; }
inline PerThreadValue PerThread(std::size_t v) { return PerThreadValue{v}; }

namespace Impl {
template <class... P>
struct policy_exec { using type = DefaultExecutionSpace; };
template <class... P>
struct policy_exec<OpenMP, P...> { using type = OpenMP; };
template <class... P>
struct policy_exec<Serial, P...> { using type = Serial; };
template <class X, class... P>
struct policy_exec<X, P...> : policy_exec<P...> {};
}  // namespace Impl

/// One team = one host thread.
class HostTeamMember {
 public:
  using execution_space = OpenMP;
  using scratch_memory_space = ScratchMemorySpace;
  HostTeamMember(int league_rank, int league_size, char* s0, std::size_t n0, char* s1,
                 std::size_t n1)
      : league_rank_(league_rank), league_size_(league_size), scr0_(s0, n0), scr1_(s1, n1) {}
  int league_rank() const { return league_rank_; }
  int league_size() const { return league_size_; }
  int team_rank() const { return 0; }
  int team_size() const { return 1; }
  void team_barrier() const {}
  ScratchMemorySpace& team_scratch(int level) const { return level == 0 ? scr0_ : scr1_; }
  ScratchMemorySpace& thread_scratch(int level) const { return level == 0 ? scr0_ : scr1_; }
  template <class T>
  void team_broadcast(T&, int) const {}
  template <class T>
  T team_broadcast(const T& v, int) const { return v; }

 private:
  int league_rank_;
  int league_size_;
  mutable ScratchMemorySpace scr0_;
  mutable ScratchMemorySpace scr1_;
};

template <class... P>
class TeamPolicy {
 public:
  using execution_space = typename Impl::policy_exec<P...>::type;
  using member_type = HostTeamMember;
  TeamPolicy(int league, AUTO_t, int = 1) : league_(league) {}
  TeamPolicy(int league, AUTO_t, AUTO_t) : league_(league) {}
  TeamPolicy(int league, int, int = 1) : league_(league) {}
  TeamPolicy(const execution_space&, int league, AUTO_t, int = 1) : league_(league) {}
  TeamPolicy(const execution_space&, int league, int, int = 1) : league_(league) {}
  /// The same league, chunk and scratch under another schedule or execution-space spelling.
  template <class... Q>
  TeamPolicy(const TeamPolicy<Q...>& o) : league_(o.league_size()), chunk_(o.chunk_size()) {
    scratch_[0] = o.scratch(0);
    scratch_[1] = o.scratch(1);
  }
  TeamPolicy& set_scratch_size(int level, PerTeamValue t) {
    scratch_[level] = t.value;
    return *this;
  }
  TeamPolicy& set_scratch_size(int level, PerTeamValue t, PerThreadValue th) {
    scratch_[level] = t.value + th.value;
    return *this;
  }
  TeamPolicy& set_scratch_size(int level, PerThreadValue th) {
    scratch_[level] = th.value;
    return *this;
  }
  TeamPolicy& set_chunk_size(int c) {
    chunk_ = c > 0 ? c : 1;
    return *this;
  }
  static int scratch_size_max(int) { return 1 << 30; }
  template <class F, class Tag = void>
  int team_size_max(const F&, Tag = {}) const { return 1; }
  template <class F, class Tag = void>
  int team_size_recommended(const F&, Tag = {}) const { return 1; }
  int league_size() const { return league_; }
  int team_size() const { return 1; }
  int chunk_size() const { return chunk_; }
  std::size_t scratch(int level) const { return scratch_[level]; }

 private:
  int league_;
  int chunk_ = 1;
  std::size_t scratch_[2] = {0, 0};
};

template <class... P>
class RangePolicy {
 public:
  using execution_space = typename Impl::policy_exec<P...>::type;
  RangePolicy(std::int64_t b, std::int64_t e) : b_(b), e_(e) {}
  RangePolicy(const execution_space&, std::int64_t b, std::int64_t e) : b_(b), e_(e) {}
  std::int64_t begin() const { return b_; }
  std::int64_t end() const { return e_; }

 private:
  std::int64_t b_, e_;
};

template <unsigned N>
struct Rank {};

/// A 2-D iteration space [b0, e0) x [b1, e1); the policy's Rank<2> is the only one used.
template <class... P>
class MDRangePolicy {
 public:
  using execution_space = typename Impl::policy_exec<P...>::type;
  using point = std::array<std::int64_t, 2>;
  MDRangePolicy(const point& b, const point& e) : b_(b), e_(e) {}
  MDRangePolicy(const execution_space&, const point& b, const point& e) : b_(b), e_(e) {}
  const point& lower() const { return b_; }
  const point& upper() const { return e_; }

 private:
  point b_, e_;
};

template <class Member>
struct TeamThreadRangeBoundaries {
  int start;
  int end;
};
template <class Member>
TeamThreadRangeBoundaries<Member> TeamThreadRange(const Member&, int n) { return {0, n}; }
template <class Member>
TeamThreadRangeBoundaries<Member> TeamThreadRange(const Member&, int b, int e) { return {b, e}; }
template <class Member>
TeamThreadRangeBoundaries<Member> ThreadVectorRange(const Member&, int n) { return {0, n}; }
template <class Member>
TeamThreadRangeBoundaries<Member> ThreadVectorRange(const Member&, int b, int e) { return {b, e}; }
template <class Member>
TeamThreadRangeBoundaries<Member> TeamVectorRange(const Member&, int n) { return {0, n}; }
template <class Member>
TeamThreadRangeBoundaries<Member> TeamVectorRange(const Member&, int b, int e) { return {b, e}; }

template <class Member>
struct SingleTeam { const Member& m; };
template <class Member>
SingleTeam<Member> PerTeam(const Member& m) { return SingleTeam<Member>{m}; }
template <class Member, class F>
void single(const SingleTeam<Member>&, const F& f) { f(); }
template <class Member, class F, class T>
void single(const SingleTeam<Member>&, const F& f, T& v) { f(v); }

// ---------------------------------------------------------------- dispatch
template <class Member, class F>
void parallel_for(const TeamThreadRangeBoundaries<Member>& r, const F& f) {
  for (int i = r.start; i < r.end; ++i) f(i);
}
template <class Member, class F, class T>
void parallel_reduce(const TeamThreadRangeBoundaries<Member>& r, const F& f, T& result) {
  T acc{};
  for (int i = r.start; i < r.end; ++i) f(i, acc);
  result = acc;
}

namespace Impl {
inline bool nested() { return omp_in_parallel() != 0 || omp_get_level() > 0; }
}  // namespace Impl

template <class... P, class F>
void parallel_for(const std::string&, const TeamPolicy<P...>& pol, const F& f) {
  using Exec = typename TeamPolicy<P...>::execution_space;
  const int n = pol.league_size();
  const std::size_t s0 = pol.scratch(0), s1 = pol.scratch(1);
  const bool par = Exec::kParallel && !Impl::nested();
  const int chunk = pol.chunk_size();
#pragma omp parallel if (par)
  {
    std::vector<char> b0(s0 + 64), b1(s1 + 64);
#pragma omp for schedule(dynamic, chunk)
    for (int i = 0; i < n; ++i) {
      HostTeamMember m(i, n, b0.data(), s0 + 64, b1.data(), s1 + 64);
      f(m);
    }
  }
}
template <class... P, class F>
void parallel_for(const TeamPolicy<P...>& pol, const F& f) { parallel_for(std::string(), pol, f); }

template <class... P, class F>
void parallel_for(const std::string&, const RangePolicy<P...>& pol, const F& f) {
  using Exec = typename RangePolicy<P...>::execution_space;
  const bool par = Exec::kParallel && !Impl::nested();
  const std::int64_t b = pol.begin(), e = pol.end();
#pragma omp parallel for if (par) schedule(static)
  for (std::int64_t i = b; i < e; ++i) f(static_cast<int>(i));
}
template <class... P, class F>
void parallel_for(const RangePolicy<P...>& pol, const F& f) { parallel_for(std::string(), pol, f); }
template <class... P, class F>
void parallel_for(const std::string&, const MDRangePolicy<P...>& pol, const F& f) {
  using Exec = typename MDRangePolicy<P...>::execution_space;
  const bool par = Exec::kParallel && !Impl::nested();
  const std::int64_t b0 = pol.lower()[0], e0 = pol.upper()[0];
  const std::int64_t b1 = pol.lower()[1], e1 = pol.upper()[1];
#pragma omp parallel for if (par) schedule(static)
  for (std::int64_t i = b0; i < e0; ++i)
    for (std::int64_t j = b1; j < e1; ++j) f(static_cast<int>(i), static_cast<int>(j));
}
template <class... P, class F>
void parallel_for(const MDRangePolicy<P...>& pol, const F& f) {
  parallel_for(std::string(), pol, f);
}
template <class F>
void parallel_for(const std::string& label, std::size_t n, const F& f) {
  parallel_for(label, RangePolicy<>(0, static_cast<std::int64_t>(n)), f);
}
template <class F>
void parallel_for(std::size_t n, const F& f) {
  parallel_for(std::string(), RangePolicy<>(0, static_cast<std::int64_t>(n)), f);
}

// ---------------------------------------------------------------- math
template <class T>
KOKKOS_INLINE_FUNCTION constexpr T max(const T& a, const T& b) { return (a < b) ? b : a; }
template <class T>
KOKKOS_INLINE_FUNCTION constexpr T min(const T& a, const T& b) { return (b < a) ? b : a; }
inline float abs(float x) { return std::fabs(x); }
inline double abs(double x) { return std::fabs(x); }
inline int abs(int x) { return std::abs(x); }
inline float fabs(float x) { return std::fabs(x); }
inline double fabs(double x) { return std::fabs(x); }
#define WW_COMPAT_UNARY(NAME)                          \
  inline float NAME(float x) { return std::NAME(x); }  \
  inline double NAME(double x) { return std::NAME(x); }
WW_COMPAT_UNARY(sqrt)
WW_COMPAT_UNARY(cbrt)
WW_COMPAT_UNARY(exp)
WW_COMPAT_UNARY(exp2)
WW_COMPAT_UNARY(expm1)
WW_COMPAT_UNARY(log)
WW_COMPAT_UNARY(log10)
WW_COMPAT_UNARY(log2)
WW_COMPAT_UNARY(log1p)
WW_COMPAT_UNARY(sin)
WW_COMPAT_UNARY(cos)
WW_COMPAT_UNARY(tan)
WW_COMPAT_UNARY(asin)
WW_COMPAT_UNARY(acos)
WW_COMPAT_UNARY(atan)
WW_COMPAT_UNARY(sinh)
WW_COMPAT_UNARY(cosh)
WW_COMPAT_UNARY(tanh)
WW_COMPAT_UNARY(asinh)
WW_COMPAT_UNARY(acosh)
WW_COMPAT_UNARY(atanh)
WW_COMPAT_UNARY(floor)
WW_COMPAT_UNARY(ceil)
WW_COMPAT_UNARY(round)
WW_COMPAT_UNARY(trunc)
WW_COMPAT_UNARY(erf)
WW_COMPAT_UNARY(erfc)
#undef WW_COMPAT_UNARY
inline float pow(float x, float y) { return std::pow(x, y); }
inline double pow(double x, double y) { return std::pow(x, y); }
inline float atan2(float y, float x) { return std::atan2(y, x); }
inline double atan2(double y, double x) { return std::atan2(y, x); }
inline float copysign(float x, float y) { return std::copysign(x, y); }
inline double copysign(double x, double y) { return std::copysign(x, y); }
inline float fmod(float x, float y) { return std::fmod(x, y); }
inline double fmod(double x, double y) { return std::fmod(x, y); }
inline float hypot(float x, float y) { return std::hypot(x, y); }
inline double hypot(double x, double y) { return std::hypot(x, y); }
inline bool isnan(float x) { return std::isnan(x); }
inline bool isnan(double x) { return std::isnan(x); }
inline bool isinf(float x) { return std::isinf(x); }
inline bool isinf(double x) { return std::isinf(x); }
inline bool isfinite(float x) { return std::isfinite(x); }
inline bool isfinite(double x) { return std::isfinite(x); }

template <class T>
inline constexpr T finite_max_v = std::numeric_limits<T>::max();
template <class T>
inline constexpr T finite_min_v = std::numeric_limits<T>::lowest();
template <class T>
inline constexpr T epsilon_v = std::numeric_limits<T>::epsilon();
template <class T>
inline constexpr T infinity_v = std::numeric_limits<T>::infinity();
template <class T>
inline constexpr T quiet_NaN_v = std::numeric_limits<T>::quiet_NaN();
template <class T>
inline constexpr T norm_min_v = std::numeric_limits<T>::min();
namespace Experimental {
using Kokkos::epsilon_v;
using Kokkos::finite_max_v;
using Kokkos::finite_min_v;
using Kokkos::infinity_v;
using Kokkos::norm_min_v;
using Kokkos::quiet_NaN_v;
}  // namespace Experimental

}  // namespace Kokkos
