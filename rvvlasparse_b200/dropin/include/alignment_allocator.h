// alignment_allocator.h — an allocator returning N-byte aligned storage
// (the element type of spMtxCSR5's vectors in the RVVLASparse API).
#pragma once
#include <cstddef>
#include <cstdlib>
#include <new>

template <typename T, std::size_t N = 16>
class AlignmentAllocator {
 public:
  typedef T value_type;
  typedef std::size_t size_type;
  typedef std::ptrdiff_t difference_type;
  typedef T* pointer;
  typedef const T* const_pointer;
  typedef T& reference;
  typedef const T& const_reference;
  template <typename U>
  struct rebind {
    typedef AlignmentAllocator<U, N> other;
  };

  AlignmentAllocator() noexcept {}
  template <typename U>
  AlignmentAllocator(const AlignmentAllocator<U, N>&) noexcept {}

  T* allocate(size_type count) {
    const std::size_t bytes = ((count * sizeof(T) + N - 1) / N) * N;
    void* p = std::aligned_alloc(N, bytes ? bytes : N);
    if (!p) throw std::bad_alloc();
    return static_cast<T*>(p);
  }
  void deallocate(T* p, size_type) noexcept { std::free(p); }

  template <typename U>
  bool operator==(const AlignmentAllocator<U, N>&) const noexcept { return true; }
  template <typename U>
  bool operator!=(const AlignmentAllocator<U, N>&) const noexcept { return false; }
};
