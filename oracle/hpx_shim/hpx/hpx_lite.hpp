/*
 * hpx_lite.hpp -- a serial, single-locality stand-in for the part of the HPX
 * API that the reference's tree and particle code uses (src/tree.cpp,
 * src/part_vect.cpp, tigergrav/tree.hpp under HPX_LITE).  TEST
 * INFRASTRUCTURE ONLY: it lets oracle/Makefile compile the reference's own
 * tree build and walk (refine, compute_multipoles, kick_fmm) where they lie,
 * so that the restated tree and walk of the oracle can be checked against
 * them.  Written for this repository from HPX's public interface; nothing
 * of HPX or of the reference's hpx_lite is used.
 *
 * Semantics: one locality (id 0); hpx::async runs its function at once on
 * the calling thread (launch::deferred runs it at the first get or wait);
 * futures hold their value in shared state, continuations (then) run when
 * their result is first needed; promises fill the state later; spinlocks do
 * nothing (there is one thread).  Components are heap objects named by a
 * pointer; actions call the function or member directly.
 */
#pragma once

#include <cstdint>
#include <cstdlib>
#include <functional>
#include <memory>
#include <mutex>
#include <optional>
#include <tuple>
#include <type_traits>
#include <utility>
#include <vector>

namespace hpx {

/* ---- futures ---- */
namespace detail {
template <class T>
struct state {
    std::optional<T> value;
    std::function<T()> thunk;
    T &get() {
        if (!value) {
            if (!thunk) std::abort(); /* read before the promise was kept */
            auto f = std::move(thunk);
            thunk = nullptr;
            value.emplace(f());
        }
        return *value;
    }
    bool ready() const { return value.has_value(); }
};
template <>
struct state<void> {
    bool done = false;
    std::function<void()> thunk;
    void get() {
        if (!done) {
            if (thunk) {
                auto f = std::move(thunk);
                thunk = nullptr;
                f();
            }
            done = true;
        }
    }
    bool ready() const { return done; }
};

/* a move-only callable as the copyable std::function of a state */
template <class R, class F>
std::function<R()> thunk_of(F &&f) {
    auto h = std::make_shared<std::decay_t<F>>(std::forward<F>(f));
    return [h]() -> R { return (*h)(); };
}
}  // namespace detail

template <class T>
class future;
template <class T>
class shared_future;

template <class T>
struct is_future : std::false_type {};
template <class T>
struct is_future<future<T>> : std::true_type {};
template <class T>
struct is_future<shared_future<T>> : std::true_type {};

template <class T>
class future {
    std::shared_ptr<detail::state<T>> s_;
    template <class U>
    friend class shared_future;

public:
    using result_type = T;
    future() = default;
    explicit future(std::shared_ptr<detail::state<T>> s) : s_(std::move(s)) {}
    future(future &&) = default;
    future &operator=(future &&) = default;
    future(const future &) = delete;
    future &operator=(const future &) = delete;
    bool valid() const { return (bool)s_; }
    bool is_ready() const { return s_ && s_->ready(); }
    void wait() const {
        if (s_) s_->get();
    }
    T get() {
        auto s = std::move(s_);
        if constexpr (std::is_void_v<T>) {
            s->get();
        } else {
            return std::move(s->get());
        }
    }
    template <class F>
    auto then(F &&f) {
        using R = std::invoke_result_t<F, future<T>>;
        auto st = std::make_shared<detail::state<R>>();
        auto parent = std::move(s_);
        st->thunk = detail::thunk_of<R>([parent, fn = std::forward<F>(f)]() mutable -> R { return fn(future<T>(parent)); });
        return future<R>(st);
    }
    template <class A>
    void serialize(A &&, unsigned) {}
};

template <class T>
class shared_future {
    std::shared_ptr<detail::state<T>> s_;

public:
    shared_future() = default;
    shared_future(future<T> &&f) : s_(std::move(f.s_)) {}
    shared_future &operator=(future<T> &&f) {
        s_ = std::move(f.s_);
        return *this;
    }
    bool valid() const { return (bool)s_; }
    void wait() const {
        if (s_) s_->get();
    }
    decltype(auto) get() const {
        if constexpr (std::is_void_v<T>) {
            s_->get();
        } else {
            return static_cast<const T &>(s_->get());
        }
    }
};

template <class T>
future<std::decay_t<T>> make_ready_future(T &&v) {
    auto st = std::make_shared<detail::state<std::decay_t<T>>>();
    st->value.emplace(std::forward<T>(v));
    return future<std::decay_t<T>>(st);
}
inline future<void> make_ready_future() {
    auto st = std::make_shared<detail::state<void>>();
    st->done = true;
    return future<void>(st);
}

namespace lcos {
namespace local {
template <class T>
class promise {
    std::shared_ptr<detail::state<T>> s_ = std::make_shared<detail::state<T>>();

public:
    future<T> get_future() { return future<T>(s_); }
    template <class U>
    void set_value(U &&v) {
        s_->value.emplace(std::forward<U>(v));
    }
};
template <>
class promise<void> {
    std::shared_ptr<detail::state<void>> s_ = std::make_shared<detail::state<void>>();

public:
    future<void> get_future() { return future<void>(s_); }
    void set_value() { s_->done = true; }
};
struct spinlock {
    void lock() {}
    void unlock() {}
    bool try_lock() { return true; }
};
}  // namespace local
}  // namespace lcos

namespace launch {
struct deferred_policy {};
constexpr deferred_policy deferred{};
}  // namespace launch

/* async of a callable: run now, the result in a ready future */
template <class F, class... A, class = std::enable_if_t<!std::is_same_v<std::decay_t<F>, launch::deferred_policy>>>
auto async(F &&f, A &&...a) {
    using R = std::invoke_result_t<F, A...>;
    if constexpr (std::is_void_v<R>) {
        std::invoke(std::forward<F>(f), std::forward<A>(a)...);
        return make_ready_future();
    } else {
        return make_ready_future(std::invoke(std::forward<F>(f), std::forward<A>(a)...));
    }
}
/* async with launch::deferred: run at the first get or wait */
template <class F, class... A>
auto async(launch::deferred_policy, F &&f, A &&...a) {
    using R = std::invoke_result_t<std::decay_t<F>, std::decay_t<A>...>;
    auto st = std::make_shared<detail::state<R>>();
    st->thunk = detail::thunk_of<R>([fn = std::decay_t<F>(std::forward<F>(f)),
                                     args = std::make_tuple(std::decay_t<A>(std::forward<A>(a))...)]() mutable -> R {
        return std::apply(fn, std::move(args));
    });
    return future<R>(st);
}

/* ---- localities and component ids ---- */
struct id_type {
    void *p = nullptr;
    template <class A>
    void serialize(A &&, unsigned) {}
    bool operator==(const id_type &o) const { return p == o.p; }
};
inline std::uint32_t get_locality_id() { return 0; }
inline id_type find_here() { return id_type{}; }
inline std::vector<id_type> find_all_localities() { return std::vector<id_type>(1); }
namespace naming {
inline std::uint32_t get_locality_id_from_gid(const id_type &) { return 0; }
}  // namespace naming

/* async of an action on a locality or component: the call, now; an action
 * whose function returns a future gives that future */
template <class Action, class... A>
auto async(const id_type &id, A &&...a) {
    using R = decltype(Action()(id, std::forward<A>(a)...));
    if constexpr (std::is_void_v<R>) {
        Action()(id, std::forward<A>(a)...);
        return make_ready_future();
    } else if constexpr (is_future<R>::value) {
        return Action()(id, std::forward<A>(a)...);
    } else {
        return make_ready_future(Action()(id, std::forward<A>(a)...));
    }
}

namespace components {
template <class T>
struct managed_component_base {};
template <class T>
struct managed_component {};
}  // namespace components

/* the created components, released by release_components() */
namespace detail {
inline std::vector<std::function<void()>> &component_deleters() {
    static std::vector<std::function<void()>> d;
    return d;
}
}  // namespace detail
template <class T, class... A>
future<id_type> new_(const id_type &, A &&...a) {
    T *obj = new T(std::forward<A>(a)...);
    detail::component_deleters().push_back([obj]() { delete obj; });
    return make_ready_future(id_type{obj});
}
inline void release_components() {
    for (auto &d : detail::component_deleters()) d();
    detail::component_deleters().clear();
}

/* ---- waiting ---- */
template <class It>
void wait_all(It b, It e) {
    for (; b != e; ++b) b->wait();
}
template <class T>
void wait_all(std::vector<T> &v) {
    for (auto &f : v) f.wait();
}
template <class T>
void wait_all(const std::vector<T> &v) {
    for (auto &f : v) f.wait();
}
template <class... F, class = std::enable_if_t<(is_future<std::decay_t<F>>::value && ...)>>
void wait_all(F &...f) {
    (f.wait(), ...);
}

}  // namespace hpx

/* actions: plain functions and component members called directly */
#define HPX_SHIM_PA_PICK(_1, _2, NAME, ...) NAME
#define HPX_PLAIN_ACTION(...) HPX_SHIM_PA_PICK(__VA_ARGS__, HPX_SHIM_PA2, HPX_SHIM_PA1)(__VA_ARGS__)
#define HPX_SHIM_PA1(f) HPX_SHIM_PA2(f, f##_action)
#define HPX_SHIM_PA2(f, name)                                                          \
    struct name {                                                                     \
        template <class... A>                                                         \
        decltype(auto) operator()(const hpx::id_type &, A &&...a) const {             \
            return f(std::forward<A>(a)...);                                          \
        }                                                                             \
    }
#define HPX_DEFINE_COMPONENT_DIRECT_ACTION(cls, fn)                                   \
    struct fn##_action {                                                              \
        template <class... A>                                                         \
        decltype(auto) operator()(const hpx::id_type &id, A &&...a) const {           \
            return static_cast<cls *>(id.p)->fn(std::forward<A>(a)...);               \
        }                                                                             \
    }
#define HPX_DEFINE_COMPONENT_ACTION(cls, fn) HPX_DEFINE_COMPONENT_DIRECT_ACTION(cls, fn)
#define HPX_REGISTER_ACTION(...)
#define HPX_REGISTER_ACTION_DECLARATION(...)
#define HPX_REGISTER_COMPONENT(...)
#define HPX_REGISTER_MINIMAL_COMPONENT_FACTORY(...)
