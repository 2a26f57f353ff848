// Test infrastructure only (oracle build). A single-threaded stand-in for the parts of HPX
// that the reference's host sources compiled by the probes use (src/tree.cpp, src/particles.cpp,
// src/driver.cpp, src/initialize.cpp, src/fft.cpp, src/power.cpp, src/domain.cpp),
// so that those sources compile where they lie and run in one process: every async call runs
// at once on the calling thread and returns a ready future, actions call their function
// directly (one locality), locks are std locks.  Used only by the probes in oracle/.
#pragma once
#include <algorithm>
#include <cstring>
#include <functional>
#include <memory>
#include <mutex>
#include <optional>
#include <shared_mutex>
#include <stdexcept>
#include <type_traits>
#include <utility>
#include <vector>

namespace hpx {

using id_type = int;

namespace detail {
template<class T>
struct state {
	std::optional<T> v;
};
template<>
struct state<void> {
	bool v = false;
};
}  // namespace detail

template<class T>
class future {
public:
	std::shared_ptr<detail::state<T>> s;
	future() = default;
	explicit future(std::shared_ptr<detail::state<T>> st) : s(std::move(st)) {
	}
	bool valid() const {
		return (bool) s;
	}
	bool is_ready() const {
		return s && s->v.has_value();
	}
	T get() {
		if (!is_ready()) {
			throw std::runtime_error("hpx stub: future not ready");
		}
		T r = std::move(*s->v);
		s.reset();
		return r;
	}
	template<class F>
	auto then(F&& f) -> future<std::invoke_result_t<F, future<T>>>;
};

template<>
class future<void> {
public:
	std::shared_ptr<detail::state<void>> s;
	future() = default;
	explicit future(std::shared_ptr<detail::state<void>> st) : s(std::move(st)) {
	}
	// a future of a value converts to a future of nothing (the value is dropped), as in HPX
	template<class T>
	future(future<T>&& f) {
		if (f.is_ready()) {
			s = std::make_shared<detail::state<void>>();
			s->v = true;
		}
		f.s.reset();
	}
	bool valid() const {
		return (bool) s;
	}
	bool is_ready() const {
		return s && s->v;
	}
	void get() {
		if (!is_ready()) {
			throw std::runtime_error("hpx stub: future not ready");
		}
		s.reset();
	}
	template<class F>
	auto then(F&& f) -> future<std::invoke_result_t<F, future<void>>>;
};

template<class T>
class shared_future {
public:
	std::shared_ptr<detail::state<T>> s;
	shared_future() = default;
	shared_future(future<T>&& f) : s(std::move(f.s)) {
	}
	bool valid() const {
		return (bool) s;
	}
	bool is_ready() const {
		return s && s->v.has_value();
	}
	const T& get() const {
		if (!is_ready()) {
			throw std::runtime_error("hpx stub: shared future not ready");
		}
		return *s->v;
	}
};

template<class T>
class promise {
	std::shared_ptr<detail::state<T>> s = std::make_shared<detail::state<T>>();
public:
	future<T> get_future() {
		return future<T>(s);
	}
	template<class V>
	void set_value(V&& v) {
		s->v.emplace(std::forward<V>(v));
	}
};
template<>
class promise<void> {
	std::shared_ptr<detail::state<void>> s = std::make_shared<detail::state<void>>();
public:
	future<void> get_future() {
		return future<void>(s);
	}
	void set_value() {
		s->v = true;
	}
};

template<class V>
future<std::decay_t<V>> make_ready_future(V&& v) {
	auto st = std::make_shared<detail::state<std::decay_t<V>>>();
	st->v.emplace(std::forward<V>(v));
	return future<std::decay_t<V>>(st);
}
inline future<void> make_ready_future() {
	auto st = std::make_shared<detail::state<void>>();
	st->v = true;
	return future<void>(st);
}

namespace detail {
template<class F, class... A>
auto run(F&& f, A&&... a) {
	using R = std::invoke_result_t<F, A...>;
	if constexpr (std::is_void_v<R>) {
		std::invoke(std::forward<F>(f), std::forward<A>(a)...);
		return make_ready_future();
	} else {
		return make_ready_future(std::invoke(std::forward<F>(f), std::forward<A>(a)...));
	}
}
struct executor_tag {
};
}  // namespace detail

template<class T>
template<class F>
auto future<T>::then(F&& f) -> future<std::invoke_result_t<F, future<T>>> {
	return detail::run(std::forward<F>(f), std::move(*this));
}
template<class F>
auto future<void>::then(F&& f) -> future<std::invoke_result_t<F, future<void>>> {
	return detail::run(std::forward<F>(f), std::move(*this));
}

namespace threads {
enum class thread_priority {
	normal, high
};
}
namespace execution {
struct parallel_executor : detail::executor_tag {
	parallel_executor() = default;
	explicit parallel_executor(threads::thread_priority) {
	}
};
struct task_policy_tag {
};
inline constexpr task_policy_tag task { };
struct par_policy {
	par_policy operator()(task_policy_tag) const {
		return *this;
	}
};
inline constexpr par_policy par { };
}  // namespace execution

// hpx::async(f, args...), hpx::async(executor, f, args...), hpx::async<Action>(locality, args...)
template<class F, class... A, std::enable_if_t<!std::is_base_of_v<detail::executor_tag, std::decay_t<F>>, int> = 0>
auto async(F&& f, A&&... a) {
	return detail::run(std::forward<F>(f), std::forward<A>(a)...);
}
template<class E, class F, class... A, std::enable_if_t<std::is_base_of_v<detail::executor_tag, std::decay_t<E>>, int> = 0>
auto async(E&&, F&& f, A&&... a) {
	return detail::run(std::forward<F>(f), std::forward<A>(a)...);
}
template<class Action, class... A>
auto async(id_type, A&&... a) {
	return detail::run(Action(), std::forward<A>(a)...);
}
template<class F, class... A>
void apply(F&& f, A&&... a) {
	std::invoke(std::forward<F>(f), std::forward<A>(a)...);
}
template<class Action, class... A>
void apply(id_type, A&&... a) {
	Action()(std::forward<A>(a)...);
}

template<class It>
void wait_all(It b, It e) {
	for (; b != e; ++b) {
		if (b->valid() && !b->is_ready()) {
			throw std::runtime_error("hpx stub: waiting on a future that is not ready");
		}
	}
}
template<class T>
void wait_all(std::vector<T>& v) {
	wait_all(v.begin(), v.end());
}
template<class T>
void wait_all(std::vector<T>&& v) {
	wait_all(v.begin(), v.end());
}

template<class P, class It, class O>
future<void> copy(P, It b, It e, O d) {
	std::copy(b, e, d);
	return make_ready_future();
}
template<class P, class It, class V>
future<void> fill(P, It b, It e, const V& v) {
	std::fill(b, e, v);
	return make_ready_future();
}
template<class P, class It, class C>
future<void> sort(P, It b, It e, C c) {
	std::sort(b, e, c);
	return make_ready_future();
}
template<class P, class It>
future<void> sort(P, It b, It e) {
	std::sort(b, e);
	return make_ready_future();
}

using mutex = std::mutex;
using spinlock = std::mutex;
using shared_mutex = std::shared_mutex;

inline void this_thread_yield() {
}
}  // namespace hpx

// an action calls its function directly (one locality); HPX_PLAIN_ACTION(f) names it f_action,
// HPX_PLAIN_ACTION(f, name) names it name
#define HPX_PLAIN_ACTION_NAMED(f, name)                                       \
	struct name {                                                               \
		template<class... A>                                                    \
		auto operator()(A&&... a) const -> decltype(f(std::forward<A>(a)...)) { \
			return f(std::forward<A>(a)...);                                      \
		}                                                                       \
	}
#define HPX_PLAIN_ACTION_1(f) HPX_PLAIN_ACTION_NAMED(f, f##_action)
#define HPX_PLAIN_ACTION_PICK(_1, _2, which, ...) which
#define HPX_PLAIN_ACTION(...) HPX_PLAIN_ACTION_PICK(__VA_ARGS__, HPX_PLAIN_ACTION_NAMED, HPX_PLAIN_ACTION_1, unused)(__VA_ARGS__)
