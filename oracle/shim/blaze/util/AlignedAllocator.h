// Stand-in for blaze::AlignedAllocator (test infrastructure for the oracle; see ../Math.h).
// blazeRT only uses it as the allocator of std::vector (blazert/datatypes.h:53-59); with the
// unpadded, unaligned vector types it selects, plain new/delete storage behaves the same.
#pragma once
#ifndef BZR_ORACLE_BLAZE_SHIM_ALIGNED_ALLOCATOR_H_
#define BZR_ORACLE_BLAZE_SHIM_ALIGNED_ALLOCATOR_H_

#include <cstddef>
#include <new>

namespace blaze {

template <typename Type>
class AlignedAllocator {
 public:
  using value_type = Type;
  AlignedAllocator() noexcept = default;
  template <typename U>
  AlignedAllocator(const AlignedAllocator<U> &) noexcept {}
  Type *allocate(std::size_t n) {
    return static_cast<Type *>(::operator new(n * sizeof(Type), std::align_val_t(64)));
  }
  void deallocate(Type *p, std::size_t) noexcept { ::operator delete(p, std::align_val_t(64)); }
  template <typename U>
  bool operator==(const AlignedAllocator<U> &) const noexcept { return true; }
  template <typename U>
  bool operator!=(const AlignedAllocator<U> &) const noexcept { return false; }
};

}  // namespace blaze

#endif  // BZR_ORACLE_BLAZE_SHIM_ALIGNED_ALLOCATOR_H_
