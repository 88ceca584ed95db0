/* Build-compatibility header for compiling the reference CPU code with GCC 13.
 *
 * Test infrastructure only, force-included (-include) by oracle/Makefile when
 * it compiles the reference sources in place; nothing here changes what the
 * reference computes.
 *
 * 1. The reference uses std::mt19937 without including <random>
 *    (src/base/misc.hh:179-188).
 * 2. Fourier::FFT_allocator (src/base/fft.hh:18-42) derives from
 *    std::allocator<T> and inherits its `rebind`, which GCC 13's
 *    allocator_traits rejects with a static_assert. The specialisation below
 *    gives the allocator the traits it was written to have (rebinding to
 *    itself); allocation still goes through the reference's own
 *    allocate/deallocate, i.e. through fftw_malloc/fftw_free.
 */
#pragma once
#include <random>
#include <memory>
#include <limits>
#include <type_traits>

namespace Fourier {
template <typename T> class FFT_allocator;
}

namespace std {
template <typename T> struct allocator_traits<Fourier::FFT_allocator<T>> {
    typedef Fourier::FFT_allocator<T> allocator_type;
    typedef T value_type;
    typedef T *pointer;
    typedef const T *const_pointer;
    typedef void *void_pointer;
    typedef const void *const_void_pointer;
    typedef std::ptrdiff_t difference_type;
    typedef std::size_t size_type;
    typedef std::false_type propagate_on_container_copy_assignment;
    typedef std::false_type propagate_on_container_move_assignment;
    typedef std::false_type propagate_on_container_swap;
    typedef std::true_type is_always_equal;

    template <typename U> using rebind_alloc = Fourier::FFT_allocator<U>;
    template <typename U> using rebind_traits = allocator_traits<Fourier::FFT_allocator<U>>;

    static pointer allocate(allocator_type &a, size_type n) { return a.allocate(n); }
    static void deallocate(allocator_type &a, pointer p, size_type n) { a.deallocate(p, n); }
    template <typename U, typename... Args>
    static void construct(allocator_type &, U *p, Args &&...args) {
        ::new ((void *)p) U(std::forward<Args>(args)...);
    }
    template <typename U> static void destroy(allocator_type &, U *p) { p->~U(); }
    static size_type max_size(const allocator_type &) {
        return std::numeric_limits<size_type>::max() / sizeof(T);
    }
    static allocator_type select_on_container_copy_construction(const allocator_type &a) {
        return a;
    }
};
}  // namespace std
