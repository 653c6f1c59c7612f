// cmm_multiply: command-line front end over libcmm_b200.so with the
// options of the reference's `multiply` program (multiply.cpp:44-243):
//
//   cmm_multiply [-f] [-a gemm|fft|fwht] [-b B] [-d D] [-v]... A.npy B.npy C.npy
//
// A.npy holds AT (n_inner x n_a), B.npy holds B (n_inner x n_b), both
// float64 (C or Fortran order); C.npy receives C = AT^T B (n_a x n_b,
// float64, C order): exact for gemm, the compressed estimate for fft / fwht
// (multiply-add-shift hashing as the reference).  Extensions: --seed S fixes
// the hash seed (otherwise drawn from the clock as the reference does),
// --hash selects the family.  Inputs are read into pinned host memory so
// the copies to the device run at full speed.  Errors print
// "<argv0>: error: <message>" and exit with status 1.
#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <stdexcept>
#include <string>
#include <sys/stat.h>
#include <vector>

#include "../../include/compmatmul_b200.h"

namespace {

struct Npy {
  std::vector<size_t> shape;
  bool fortran = false;
  size_t word = 0;
  std::string descr;
  double* data = nullptr;  // pinned host memory
  size_t count = 0;
  ~Npy() {
    if (data) cudaFreeHost(data);
  }
};

std::string field(const std::string& hdr, const std::string& key) {
  const size_t k = hdr.find("'" + key + "'");
  if (k == std::string::npos) throw std::runtime_error("malformed .npy header (no " + key + ")");
  size_t v = hdr.find(':', k);
  if (v == std::string::npos) throw std::runtime_error("malformed .npy header");
  ++v;
  while (v < hdr.size() && hdr[v] == ' ') ++v;
  return hdr.substr(v);
}

void load_npy(const std::string& path, Npy& out, const char* name) {
  std::ifstream f(path, std::ios::binary);
  if (!f) throw std::runtime_error("cannot open `" + path + "'");
  char magic[8];
  f.read(magic, 8);
  if (!f || std::memcmp(magic, "\x93NUMPY", 6) != 0) throw std::runtime_error("`" + path + "' is not a .npy file");
  const int major = (unsigned char)magic[6];
  uint32_t hlen = 0;
  if (major == 1) {
    unsigned char h[2];
    f.read(reinterpret_cast<char*>(h), 2);
    hlen = h[0] | (h[1] << 8);
  } else {
    unsigned char h[4];
    f.read(reinterpret_cast<char*>(h), 4);
    hlen = h[0] | (h[1] << 8) | (h[2] << 16) | ((uint32_t)h[3] << 24);
  }
  std::string hdr(hlen, '\0');
  f.read(&hdr[0], hlen);
  if (!f) throw std::runtime_error("truncated .npy header in `" + path + "'");
  // descr: '<f8'
  std::string d = field(hdr, "descr");
  if (d.size() < 3 || d[0] != '\'') throw std::runtime_error("malformed .npy descr");
  out.descr = d.substr(1, d.find('\'', 1) - 1);
  size_t digits = out.descr.find_first_of("0123456789");
  out.word = digits == std::string::npos ? 0 : (size_t)std::atoi(out.descr.c_str() + digits);
  out.fortran = field(hdr, "fortran_order").compare(0, 4, "True") == 0;
  std::string s = field(hdr, "shape");
  const size_t open = s.find('('), close = s.find(')');
  if (open == std::string::npos || close == std::string::npos) throw std::runtime_error("malformed .npy shape");
  std::string dims = s.substr(open + 1, close - open - 1);
  size_t pos = 0;
  while (pos < dims.size()) {
    while (pos < dims.size() && (dims[pos] == ' ' || dims[pos] == ',')) ++pos;
    if (pos >= dims.size()) break;
    out.shape.push_back((size_t)std::strtoull(dims.c_str() + pos, nullptr, 10));
    while (pos < dims.size() && dims[pos] != ',') ++pos;
  }
  if (out.shape.size() != 2)
    throw std::runtime_error(std::string("Dimension mismatch: ") + name + " has " + std::to_string(out.shape.size()) +
                             " dims, but 2 expected!");
  if (out.word != sizeof(double))
    throw std::runtime_error(std::string("Word size mismatch: ") + name + " is expected to have word size of " +
                             std::to_string(sizeof(double)) + ", but got " + std::to_string(out.word));
  if (out.descr != "<f8" && out.descr != "=f8")
    throw std::runtime_error(std::string(name) + " is expected to hold little-endian float64 values (got '" +
                             out.descr + "')");
  out.count = out.shape[0] * out.shape[1];
  if (cudaMallocHost(reinterpret_cast<void**>(&out.data), std::max<size_t>(out.count, 1) * 8) != cudaSuccess) {
    out.data = nullptr;
    throw std::runtime_error("cannot allocate pinned host memory");
  }
  f.read(reinterpret_cast<char*>(out.data), (std::streamsize)(out.count * 8));
  if (!f) throw std::runtime_error("truncated data in `" + path + "'");
}

// Fortran (column-major) rows x cols -> C order, in place through a copy
void fortran_to_c(Npy& a) {
  const size_t rows = a.shape[0], cols = a.shape[1];
  std::vector<double> tmp(a.data, a.data + a.count);
  for (size_t i = 0; i < rows; ++i)
    for (size_t j = 0; j < cols; ++j) a.data[i * cols + j] = tmp[j * rows + i];
}

void save_npy(const std::string& path, const double* c, size_t rows, size_t cols) {
  std::string dict = "{'descr': '<f8', 'fortran_order': False, 'shape': (" + std::to_string(rows) + ", " +
                     std::to_string(cols) + "), }";
  size_t total = 10 + dict.size() + 1;
  const size_t pad = (64 - total % 64) % 64;
  dict += std::string(pad, ' ') + "\n";
  std::ofstream f(path, std::ios::binary | std::ios::trunc);
  if (!f) throw std::runtime_error("cannot write `" + path + "'");
  const uint16_t hl = (uint16_t)dict.size();
  f.write("\x93NUMPY\x01\x00", 8);
  const unsigned char h[2] = {(unsigned char)(hl & 0xff), (unsigned char)(hl >> 8)};
  f.write(reinterpret_cast<const char*>(h), 2);
  f.write(dict.data(), (std::streamsize)dict.size());
  f.write(reinterpret_cast<const char*>(c), (std::streamsize)(rows * cols * 8));
  if (!f) throw std::runtime_error("write failed for `" + path + "'");
}

void usage(const char* argv0) {
  std::fprintf(stderr,
               "usage: %s [-f] [-a gemm|fft|fwht] [-b B] [-d D] [--seed S] [--hash H] [-v]... "
               "<A.npy> <B.npy> <C.npy>\n"
               "Computes C = A^T B: A.npy holds AT (inner x n_a), B.npy holds B (inner x n_b).\n"
               "  -f, --force      overwrite C.npy\n"
               "  -a, --algorithm  gemm (exact, default), fft or fwht (compressed)\n"
               "  -b, --buckets    buckets per sketch (power of 2; fft / fwht)\n"
               "  -d, --sketches   number of sketches (positive; fft / fwht)\n"
               "  --seed S         hash seed (default: drawn from the clock)\n"
               "  --hash H         multiply-shift | multiply-add-shift (default) | tabulation8 | tabulation16\n"
               "  -v, --verbose    more output (repeatable)\n",
               argv0);
}

void check(int st) {
  if (st != CMM_OK) throw std::runtime_error(cmm_last_error());
}

}  // namespace

int main(int argc, char* argv[]) {
  const char* argv0 = argv[0];
  try {
    std::vector<std::string> pos;
    bool force = false, b_set = false, d_set = false, has_seed = false;
    int verbose = 0, b = -1, d = -1, kind = CMM_HASH_MULTIPLY_ADD_SHIFT;
    uint64_t seed = 0;
    std::string algo = "gemm";
    for (int i = 1; i < argc; ++i) {
      const std::string a = argv[i];
      auto need = [&](const std::string& opt) -> std::string {
        if (i + 1 >= argc) throw std::runtime_error("missing value for " + opt);
        return argv[++i];
      };
      if (a == "-h" || a == "--help") {
        usage(argv0);
        return EXIT_SUCCESS;
      } else if (a == "-f" || a == "--force") {
        force = true;
      } else if (a == "-a" || a == "--algorithm") {
        algo = need(a);
        if (algo != "gemm" && algo != "fft" && algo != "fwht")
          throw std::runtime_error("Value '" + algo + "' does not meet constraint: gemm|fft|fwht");
      } else if (a == "-b" || a == "--buckets") {
        b = std::atoi(need(a).c_str());
        b_set = true;
      } else if (a == "-d" || a == "--sketches") {
        d = std::atoi(need(a).c_str());
        d_set = true;
      } else if (a == "--seed") {
        seed = std::strtoull(need(a).c_str(), nullptr, 10);
        has_seed = true;
      } else if (a == "--hash") {
        const std::string h = need(a);
        if (h == "multiply-shift") kind = CMM_HASH_MULTIPLY_SHIFT;
        else if (h == "multiply-add-shift") kind = CMM_HASH_MULTIPLY_ADD_SHIFT;
        else if (h == "tabulation8") kind = CMM_HASH_TABULATION8;
        else if (h == "tabulation16") kind = CMM_HASH_TABULATION16;
        else throw std::runtime_error("unknown hash `" + h + "'");
      } else if (a == "-v" || a == "--verbose") {
        ++verbose;
      } else if (a.size() > 1 && a[0] == '-' && a.find_first_not_of('v', 1) == std::string::npos) {
        verbose += (int)a.size() - 1;  // -vv
      } else if (!a.empty() && a[0] == '-') {
        throw std::runtime_error("unknown option `" + a + "'");
      } else {
        pos.push_back(a);
      }
    }
    if (pos.size() != 3) {
      usage(argv0);
      throw std::runtime_error("expected <A.npy> <B.npy> <C.npy>");
    }
    struct stat st;
    if (stat(pos[2].c_str(), &st) == 0 && !force) {
      std::fprintf(stderr, "%s: error: file `%s' already exists!\n", argv0, pos[2].c_str());
      return EXIT_FAILURE;
    }
    if (algo != "gemm") {
      if (!b_set) throw std::runtime_error("Got algorithm `" + algo + "' but the parameter b is not set!");
      if (b < 1 || (b & (b - 1)) != 0)
        throw std::runtime_error("The parameter b must be a positive power of 2 (got " + std::to_string(b) + ")");
      if (!d_set) throw std::runtime_error("Got algorithm `" + algo + "' but the parameter d is not set!");
      if (d < 1) throw std::runtime_error("The parameter d must be positive (got " + std::to_string(d) + ")");
    }
    Npy A, B;
    load_npy(pos[0], A, "A");
    const size_t q = A.shape[0], p = A.shape[1];
    if (A.fortran) {
      if (verbose > 0) std::fprintf(stderr, "A was given in Fortran order, converting to C order\n");
      fortran_to_c(A);
    }
    load_npy(pos[1], B, "B");
    if (B.shape[0] != q)
      throw std::runtime_error("Dimension mismatch: B is expected to have " + std::to_string(q) + " rows, but got " +
                               std::to_string(B.shape[0]) + " instead");
    const size_t r = B.shape[1];
    if (B.fortran) {
      if (verbose > 0) std::fprintf(stderr, "B was given in Fortran order, converting to C order\n");
      fortran_to_c(B);
    }
    if (verbose > 0)
      std::fprintf(stderr, "A = %s (%zu x %zu)\nB = %s (%zu x %zu)\nC = %s\nalgorithm: %s, b = %d, d = %d\n",
                   pos[0].c_str(), q, p, pos[1].c_str(), q, r, pos[2].c_str(), algo.c_str(), b, d);
    double* C = nullptr;
    if (cudaMallocHost(reinterpret_cast<void**>(&C), std::max<size_t>(p * r, 1) * 8) != cudaSuccess)
      throw std::runtime_error("cannot allocate pinned host memory");
    struct Free {
      double* p;
      ~Free() { cudaFreeHost(p); }
    } guard{C};
    if (algo == "gemm") {
      check(cmm_gemm((int64_t)p, (int64_t)q, (int64_t)r, C, A.data, B.data));
    } else {
      check(cmm_matmul(algo == "fft" ? CMM_VARIANT_FFT : CMM_VARIANT_FWHT, kind, (int64_t)p, (int64_t)q, (int64_t)r, C,
                       A.data, B.data, d, b, has_seed ? 1 : 0, seed));
    }
    if (verbose > 0) std::fprintf(stderr, "Saving result to %s\n", pos[2].c_str());
    save_npy(pos[2], C, p, r);
  } catch (const std::exception& e) {
    std::fprintf(stderr, "%s: error: %s\n", argv0, e.what());
    return EXIT_FAILURE;
  }
  return EXIT_SUCCESS;
}
