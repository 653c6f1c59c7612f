// compmatmul_module.cpp -- the drop-in for the reference's pybind11 module
// `compmatmul` (compmatmul.cpp:189-209).  Same functions, argument names,
// defaults, argument checks, messages and exception types; the work is done
// on the GPU through the C ABI of libcmm_b200.so.
//
//   gemm(C, AT, B)                                  compmatmul.cpp:76-85
//   matmul_fft(C, AT, B, d, b, seed=None, hash=None)  compmatmul.cpp:107-147
//   matmul_fwht(C, AT, B, d, b, seed=None, hash=None) compmatmul.cpp:149-186
#include <pybind11/numpy.h>
#include <pybind11/pybind11.h>
#include <pybind11/stl.h>

#include <cstdint>
#include <new>
#include <optional>
#include <stdexcept>
#include <string>

#include "compmatmul_b200.h"

namespace py = pybind11;

namespace {

// compmatmul.cpp:13-74, in the same order
void check_array_arguments(py::array C, py::array AT, py::array B) {
  py::buffer_info C_info = C.request();
  py::buffer_info AT_info = AT.request();
  py::buffer_info B_info = B.request();
  const char* dtype_msg = "compmatmul only supports double precision floats for now";
  if (!C.dtype().is(py::dtype::of<double>())) throw std::invalid_argument(dtype_msg);
  if (!AT.dtype().is(py::dtype::of<double>())) throw std::invalid_argument(dtype_msg);
  if (!B.dtype().is(py::dtype::of<double>())) throw std::invalid_argument(dtype_msg);
  if (C_info.ndim != 2)
    throw std::invalid_argument("C must have ndim=2 (got " + std::to_string(C_info.ndim) + ")");
  if (AT_info.ndim != 2)
    throw std::invalid_argument("AT must have ndim=2 (got " + std::to_string(AT_info.ndim) + ")");
  if (B_info.ndim != 2)
    throw std::invalid_argument("B must have ndim=2 (got " + std::to_string(B_info.ndim) + ")");
  const auto C_CONTIGUOUS = py::detail::npy_api::constants::NPY_ARRAY_C_CONTIGUOUS_;
  if ((C.flags() & C_CONTIGUOUS) != C_CONTIGUOUS)
    throw std::invalid_argument("The arrays must be C-contiguous");
  if ((AT.flags() & C_CONTIGUOUS) != C_CONTIGUOUS)
    throw std::invalid_argument("The arrays must be C-contiguous");
  if ((B.flags() & C_CONTIGUOUS) != C_CONTIGUOUS)
    throw std::invalid_argument("The arrays must be C-contiguous");
  const auto q = AT.shape(0), p = AT.shape(1), r = B.shape(1);
  if (B.shape(0) != q || C.shape(0) != p || C.shape(1) != r)
    throw std::invalid_argument("Shape mismatch! Note that AT is assumed to be transposed");
  if (reinterpret_cast<uintptr_t>(AT.data()) % 64 != 0)
    throw std::invalid_argument("AT is not aligned at a 64-byte boundary!");
  if (reinterpret_cast<uintptr_t>(B.data()) % 64 != 0)
    throw std::invalid_argument("B is not aligned at a 64-byte boundary!");
  if (reinterpret_cast<uintptr_t>(C.data()) % 64 != 0)
    throw std::invalid_argument("C is not aligned at a 64-byte boundary!");
}

// compmatmul.cpp:87-105
void check_other_arguments(int d, int b, const std::optional<std::string>& hash) {
  if (b < 2 || (b & (b - 1)) != 0)
    throw std::invalid_argument("b must be power of 2 greater than 1 (got " + std::to_string(b) + ")");
  if (d < 1) throw std::invalid_argument("d must be positive (got " + std::to_string(d) + ")");
  if (hash) {
    if (*hash != "multiply shift" && *hash != "multiply add shift" && *hash != "tabulation8" &&
        *hash != "tabulation16")
      throw std::invalid_argument("Invalid hash `" + *hash +
                                  "' provided; hash must be one of `multiply shift', "
                                  "`multiply add shift', `tabulation8', or `tabulation16'");
  }
}

// compmatmul.cpp:120-145: None -> multiply_add_shift_hash
int hash_kind(const std::optional<std::string>& hash) {
  if (!hash || *hash == "multiply add shift") return CMM_HASH_MULTIPLY_ADD_SHIFT;
  if (*hash == "multiply shift") return CMM_HASH_MULTIPLY_SHIFT;
  if (*hash == "tabulation8") return CMM_HASH_TABULATION8;
  if (*hash == "tabulation16") return CMM_HASH_TABULATION16;
  throw std::runtime_error("Tried to use an invalid hash");
}

// C ABI status -> the reference's exception types
void raise_status(int st) {
  if (st == CMM_OK) return;
  const std::string msg = cmm_last_error();
  switch (st) {
    case CMM_ERR_INVALID_ARGUMENT: throw std::invalid_argument(msg);
    case CMM_ERR_NO_MEMORY: throw std::bad_alloc();
    default: throw std::runtime_error(msg);
  }
}

void gemm(py::array C, py::array AT, py::array B) {
  check_array_arguments(C, AT, B);
  const int64_t q = AT.shape(0), p = AT.shape(1), r = B.shape(1);
  double* c = static_cast<double*>(C.mutable_data());
  const double* at = static_cast<const double*>(AT.data());
  const double* bb = static_cast<const double*>(B.data());
  int st;
  {
    py::gil_scoped_release nogil;
    st = cmm_gemm(p, q, r, c, at, bb);
  }
  raise_status(st);
}

void matmul_variant(int variant, py::array C, py::array AT, py::array B, int d, int b,
                    std::optional<uint64_t> seed, std::optional<std::string> hash) {
  check_array_arguments(C, AT, B);
  check_other_arguments(d, b, hash);
  const int kind = hash_kind(hash);
  const int64_t q = AT.shape(0), p = AT.shape(1), r = B.shape(1);
  double* c = static_cast<double*>(C.mutable_data());
  const double* at = static_cast<const double*>(AT.data());
  const double* bb = static_cast<const double*>(B.data());
  int st;
  {
    py::gil_scoped_release nogil;
    st = cmm_matmul(variant, kind, p, q, r, c, at, bb, d, b, seed ? 1 : 0, seed.value_or(0));
  }
  raise_status(st);
}

void matmul_fft(py::array C, py::array AT, py::array B, int d, int b,
                std::optional<uint64_t> seed = std::nullopt,
                std::optional<std::string> hash = std::nullopt) {
  matmul_variant(CMM_VARIANT_FFT, C, AT, B, d, b, seed, hash);
}

void matmul_fwht(py::array C, py::array AT, py::array B, int d, int b,
                 std::optional<uint64_t> seed = std::nullopt,
                 std::optional<std::string> hash = std::nullopt) {
  matmul_variant(CMM_VARIANT_FWHT, C, AT, B, d, b, seed, hash);
}

}  // namespace

PYBIND11_MODULE(compmatmul, m) {
  m.doc() = "Compressed Matrix Multiplication Python bindings (B200 / sm_100a)";
  m.def("gemm", &gemm,
        "Computes C = A^T B using the DGEMM function of the underlying BLAS implementation",
        py::arg("C"), py::arg("AT"), py::arg("B"));
  m.def("matmul_fft", &matmul_fft,
        "Computes C = A^T using compressed matrix multiplication with FFT", py::arg("C"),
        py::arg("AT"), py::arg("B"), py::arg("d"), py::arg("b"), py::arg("seed") = py::none(),
        py::arg("hash") = py::none());
  m.def("matmul_fwht", &matmul_fwht,
        "Computes C = A^T using compressed matrix multiplication with FWHT", py::arg("C"),
        py::arg("AT"), py::arg("B"), py::arg("d"), py::arg("b"), py::arg("seed") = py::none(),
        py::arg("hash") = py::none());
}
