// rvvla_mirror.h — the device copy a drop-in matrix object carries.
//
// Every format class of the drop-in holds one MirrorSlot.  convert() fills it
// with the GPU-built arrays (and copies them back into the class's public
// host fields); sparse_mv() uploads the host fields on first use when the slot
// is empty.  After changing a matrix's host arrays in place, call
// rvvla_dropin_reset(matrix) so the next product uploads them again.  A copy
// of a matrix starts with an empty slot; a move takes the slot along.
#pragma once
#include <memory>

namespace rvvla_dropin {

struct DeviceMirror;  // defined in the drop-in library
void release(DeviceMirror* m);

class MirrorSlot {
 public:
  MirrorSlot() = default;
  MirrorSlot(const MirrorSlot&) {}
  MirrorSlot& operator=(const MirrorSlot&) {
    ptr.reset();
    return *this;
  }
  MirrorSlot(MirrorSlot&&) = default;
  MirrorSlot& operator=(MirrorSlot&&) = default;
  DeviceMirror* get() const { return ptr.get(); }
  void set(DeviceMirror* m) const { ptr.reset(m); }
  void reset() const { ptr.reset(); }

 private:
  struct Del {
    void operator()(DeviceMirror* m) const { release(m); }
  };
  mutable std::unique_ptr<DeviceMirror, Del> ptr;
};

}  // namespace rvvla_dropin

template <class Mtx>
void rvvla_dropin_reset(const Mtx& mat) {
  mat.rvvla_dev.reset();
}
