// CRS.h — spMtxCRS<ValT> of the RVVLASparse API (include/CRS.h:10-256 of the
// reference): host CSR arrays owned with new[]/delete[], the same public
// fields and member functions, plus the device copy used by the GPU drop-in.
#pragma once
#include <cstring>
#include <iostream>

#include "rvvla_decl.h"
#include "rvvla_mirror.h"

namespace SparseMatrixLib {

typedef char MM_typecode[4];

template <typename ValT>
class spMtxCRS {
 public:
  size_t m = 0;
  size_t n = 0;
  size_t nz = 0;
  size_t capacity = 0;
  MM_typecode matcode = {0, 0, 0, 0};
  int* Rst = nullptr;
  int* Col = nullptr;
  ValT* Val = nullptr;
  rvvla_dropin::MirrorSlot rvvla_dev;

  void freeMem() {
    delete[] Col;
    delete[] Rst;
    delete[] Val;
    Col = nullptr;
    Rst = nullptr;
    Val = nullptr;
    m = n = nz = capacity = 0;
    rvvla_dev.reset();
  }

  spMtxCRS() {}
  spMtxCRS(size_t m_, size_t n_) : m(m_), n(n_) { Rst = new int[m + 1](); }
  spMtxCRS(size_t m_, size_t n_, size_t nz_) : m(m_), n(n_), nz(nz_), capacity(nz_) {
    Rst = new int[m + 1];
    Col = new int[nz];
    Val = new ValT[nz];
  }
  spMtxCRS(size_t m_, size_t n_, size_t nz_, const int* Rst_, const int* Col_, const ValT* Val_)
      : m(m_), n(n_), nz(nz_), capacity(nz_) {
    Rst = new int[m + 1];
    std::memcpy(Rst, Rst_, (m + 1) * sizeof(int));
    Col = new int[nz];
    std::memcpy(Col, Col_, nz * sizeof(int));
    if (Val_) {
      Val = new ValT[nz];
      std::memcpy(Val, Val_, nz * sizeof(ValT));
    }
  }
  spMtxCRS(const spMtxCRS& o) : m(o.m), n(o.n), nz(o.nz), capacity(o.capacity) {
    std::memcpy(matcode, o.matcode, sizeof(MM_typecode));
    Rst = new int[m + 1];
    std::memcpy(Rst, o.Rst, (m + 1) * sizeof(int));
    Col = new int[nz];
    std::memcpy(Col, o.Col, nz * sizeof(int));
    if (o.Val) {
      Val = new ValT[nz];
      std::memcpy(Val, o.Val, nz * sizeof(ValT));
    }
  }
  spMtxCRS(spMtxCRS&& o) noexcept
      : m(o.m), n(o.n), nz(o.nz), capacity(o.capacity), Rst(o.Rst), Col(o.Col), Val(o.Val),
        rvvla_dev(std::move(o.rvvla_dev)) {
    std::memcpy(matcode, o.matcode, sizeof(MM_typecode));
    o.Rst = nullptr;
    o.Col = nullptr;
    o.Val = nullptr;
  }
  ~spMtxCRS() { freeMem(); }

  void resizeVals(size_t newNz) {
    if (newNz > capacity) {
      delete[] Col;
      delete[] Val;
      Col = new int[newNz];
      Val = new ValT[newNz];
      capacity = newNz;
    }
    nz = newNz;
    rvvla_dev.reset();
  }

  void resizeRows(size_t newM) {
    if (m != newM) {
      delete[] Rst;
      Rst = new int[newM + 1]();
      m = newM;
    }
    rvvla_dev.reset();
  }

  template <typename ValT2>
  void copyPattern(const spMtxCRS<ValT2>& source) {
    resizeRows(source.m);
    std::memcpy(Rst, source.Rst, (m + 1) * sizeof(int));
    n = source.n;
    resizeVals(source.nz);
    std::memcpy(Col, source.Col, nz * sizeof(int));
  }

  spMtxCRS& operator=(const spMtxCRS& o) {
    if (this == &o) return *this;
    spMtxCRS tmp(o);
    *this = std::move(tmp);
    return *this;
  }
  spMtxCRS& operator=(spMtxCRS&& o) noexcept {
    if (this == &o) return *this;
    delete[] Col;
    delete[] Rst;
    delete[] Val;
    m = o.m; n = o.n; nz = o.nz; capacity = o.capacity;
    std::memcpy(matcode, o.matcode, sizeof(MM_typecode));
    Rst = o.Rst; Col = o.Col; Val = o.Val;
    o.Rst = nullptr; o.Col = nullptr; o.Val = nullptr;
    rvvla_dev = std::move(o.rvvla_dev);
    return *this;
  }

  spMtxCRS extractRows(size_t begin, size_t end) const {
    const size_t cnt = (size_t)(Rst[end] - Rst[begin]);
    spMtxCRS out(end - begin, n, cnt);
    for (size_t i = 0; i <= end - begin; ++i) out.Rst[i] = Rst[begin + i] - Rst[begin];
    std::memcpy(out.Col, Col + Rst[begin], cnt * sizeof(int));
    std::memcpy(out.Val, Val + Rst[begin], cnt * sizeof(ValT));
    std::memcpy(out.matcode, matcode, sizeof(MM_typecode));
    return out;
  }

  bool operator==(const spMtxCRS& o) const {
    if (m != o.m || n != o.n || nz != o.nz) return false;
    for (size_t i = 0; i <= m; ++i)
      if (Rst[i] != o.Rst[i]) return false;
    for (size_t k = 0; k < nz; ++k)
      if (Col[k] != o.Col[k] || Val[k] != o.Val[k]) return false;
    return true;
  }

  void print_crs() const {
    std::cout << m << ' ' << nz << '\n';
    for (size_t i = 0; i < m; ++i)
      for (int k = Rst[i]; k < Rst[i + 1]; ++k) {
        std::cout << i + 1 << ' ' << Col[k] + 1;
        if (Val) std::cout << ' ' << Val[k];
        std::cout << '\n';
      }
  }

  void print_dense() const {
    for (size_t i = 0; i < m; ++i) {
      size_t c = 0;
      for (int k = Rst[i]; k < Rst[i + 1]; ++k, ++c) {
        for (; c < (size_t)Col[k]; ++c) std::cout << 0 << ' ';
        std::cout << Val[k] << ' ';
      }
      for (; c < n; ++c) std::cout << 0 << ' ';
      std::cout << '\n';
    }
    std::cout << '\n';
  }

  friend std::ostream& operator<<(std::ostream& out, const spMtxCRS& a) {
    return out << "spMtxCRS( m  = " << a.m << ", n  = " << a.n << ", nz = " << a.nz << ")";
  }
};

RVVLA_DROPIN_DECLARE_SPMV(spMtxCRS)
RVVLA_DROPIN_DECLARE_SPMV_MIXED(spMtxCRS)

}  // namespace SparseMatrixLib
