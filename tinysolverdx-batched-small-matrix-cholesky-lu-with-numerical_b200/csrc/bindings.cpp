// pybind11 module `_core`: the Python face of host_api.hpp, a drop-in for
// TinySolverDx's `_core` (reference interface: src/python/bindings.cpp:115-178).
// Every reference entry point keeps its name, keyword names, defaults, return
// shapes and exception messages; backend="cuda" runs on the B200 for every entry
// point, the solves included (the reference's solves take no backend and always
// run on the CPU). New entry points: posv_cuda_* / gesv_cuda_* return (x, info)
// from one fused GPU pass.
//
// Structure: option strings are looked up in tables; every solver entry goes
// through one template (solver_entry) that validates the stack, copies the
// operand the library overwrites, allocates the integer outputs and runs the
// library without the GIL; the float64 metric entry points are registered from
// a table of (name, operand layout, function).
#include <pybind11/numpy.h>
#include <pybind11/pybind11.h>

#include <cstring>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <vector>

#include "host_api.hpp"

namespace py = pybind11;

namespace {

using tsdx::Backend;
using tsdx::Precision;

// ------------------------------------------------------------ option strings
template <class E>
struct Option {
  const char* text;
  E value;
};
const Option<Precision> kPrecision[] = {
    {"fp32", Precision::FP32}, {"fp64", Precision::FP64}, {"fp16", Precision::FP16}, {"bf16", Precision::BF16}};
const Option<Backend> kBackend[] = {{"auto", Backend::Auto},
                                    {"naive", Backend::Naive},
                                    {"scalar", Backend::Scalar},
                                    {"simd", Backend::Simd},
                                    {"cuda", Backend::Cuda}};

// The table entry named s; otherwise ValueError "<what> must be one of <names>".
template <class E, std::size_t N>
E option(const Option<E> (&table)[N], const std::string& s, const char* what) {
  std::string names;
  for (const Option<E>& o : table) {
    if (s == o.text) return o.value;
    names += names.empty() ? o.text : std::string(", ") + o.text;
  }
  throw std::invalid_argument(std::string(what) + " must be one of " + names);
}

// ------------------------------------------------------------ array shapes
template <class S>
using Arr = py::array_t<S, py::array::c_style>;  // forcecast: any input becomes C-contiguous S
using IntArr = py::array_t<int, py::array::c_style>;

// A (batch, n, n) stack and what travels with it.
struct Stack {
  py::ssize_t batch = 0;
  int n = 0;
  int nrhs = 0;
};

Stack square_stack(const py::array& a, const char* msg) {
  if (a.ndim() != 3 || a.shape(1) != a.shape(2)) throw std::invalid_argument(msg);
  Stack s;
  s.batch = a.shape(0);
  s.n = static_cast<int>(a.shape(1));
  return s;
}
void expect_rhs(Stack& s, const py::array& b) {
  if (b.ndim() != 3 || b.shape(0) != s.batch || b.shape(1) != s.n) throw std::invalid_argument("B must be (batch, n, nrhs)");
  s.nrhs = static_cast<int>(b.shape(2));
}
void expect_pivots(const Stack& s, const py::array& piv) {
  if (piv.ndim() != 2 || piv.shape(0) != s.batch || piv.shape(1) != s.n) throw std::invalid_argument("piv must be (batch, n)");
}
void expect_vector(const py::array& A, const py::array& v, const char* name) {
  square_stack(A, "A must be (batch, n, n)");
  if (v.ndim() != 2 || v.shape(0) != A.shape(0) || v.shape(1) != A.shape(1))
    throw std::invalid_argument(std::string(name) + " must be (batch, n)");
}

// A fresh C-contiguous array with a's shape and contents: the library works in
// place, and the caller's array must stay untouched.
template <class S>
Arr<S> fresh_copy(const Arr<S>& a) {
  Arr<S> out(std::vector<py::ssize_t>(a.shape(), a.shape() + a.ndim()));
  if (a.size() > 0) std::memcpy(out.mutable_data(), a.data(), sizeof(S) * static_cast<std::size_t>(a.size()));
  return out;
}
py::array_t<int> ints(std::vector<py::ssize_t> shape) { return py::array_t<int>(std::move(shape)); }

// ------------------------------------------------------------ solver entries
// What an entry point overwrites: the input stack (factorizations) or the
// right-hand sides (solves).
enum class Writes { Stack, Rhs };

// Validates, copies the operand the library overwrites, allocates pivots/info as
// asked, runs `call(work, piv, info)` with the GIL released, and returns the
// results in the reference's order: (work[, piv][, info]) or work alone.
template <class S, Writes W, bool PIV, bool INFO, class Call>
py::object solver_entry(const Arr<S>& stack, const Arr<S>* rhs, const IntArr* piv_in, Call&& call) {
  Stack st = square_stack(stack, "expected array of shape (batch, n, n)");
  if (rhs) expect_rhs(st, *rhs);
  if (piv_in) expect_pivots(st, *piv_in);
  Arr<S> work = fresh_copy<S>(W == Writes::Stack ? stack : *rhs);
  py::array_t<int> piv = PIV ? ints({st.batch, static_cast<py::ssize_t>(st.n)}) : py::array_t<int>();
  py::array_t<int> info = INFO ? ints({st.batch}) : py::array_t<int>();
  int* pivp = PIV ? piv.mutable_data() : nullptr;
  int* infop = INFO ? info.mutable_data() : nullptr;
  S* w = work.mutable_data();
  {
    py::gil_scoped_release unlocked;
    call(st, w, pivp, infop);
  }
  if constexpr (PIV && INFO) return py::make_tuple(work, piv, info);
  else if constexpr (INFO) return py::make_tuple(work, info);
  else return std::move(work);
}

template <class S>
void bind_solvers(py::module_& m, const std::string& sfx) {
  const auto name = [&](const char* op) { return std::string(op) + "_" + sfx; };
  const auto prec = [](const std::string& s) { return option(kPrecision, s, "precision"); };
  const auto back = [](const std::string& s) { return option(kBackend, s, "backend"); };

  m.def(
      name("cholesky").c_str(),
      [=](const Arr<S>& A, const std::string& precision, const std::string& backend) {
        const Precision p = prec(precision);
        const Backend b = back(backend);
        return solver_entry<S, Writes::Stack, false, true>(A, nullptr, nullptr, [&](const Stack& s, S* a, int*, int* info) {
          tsdx::cholesky<S>(p, a, s.n, s.batch, info, b);
        });
      },
      py::arg("A"), py::arg("precision") = "fp32", py::arg("backend") = "auto");
  m.def(
      name("lu").c_str(),
      [=](const Arr<S>& A, const std::string& precision, const std::string& backend) {
        const Precision p = prec(precision);
        const Backend b = back(backend);
        return solver_entry<S, Writes::Stack, true, true>(A, nullptr, nullptr, [&](const Stack& s, S* a, int* piv, int* info) {
          tsdx::lu<S>(p, a, s.n, s.batch, piv, info, b);
        });
      },
      py::arg("A"), py::arg("precision") = "fp32", py::arg("backend") = "auto");
  m.def(
      name("cholesky_solve").c_str(),
      [=](const Arr<S>& L, const Arr<S>& B, const std::string& precision, const std::string& backend) {
        const Precision p = prec(precision);
        const Backend b = back(backend);
        const S* l = L.data();
        return solver_entry<S, Writes::Rhs, false, false>(L, &B, nullptr, [&](const Stack& s, S* x, int*, int*) {
          tsdx::cholesky_solve<S>(p, l, s.n, s.batch, x, s.nrhs, b);
        });
      },
      py::arg("L"), py::arg("B"), py::arg("precision") = "fp32", py::arg("backend") = "auto");
  m.def(
      name("lu_solve").c_str(),
      [=](const Arr<S>& LU, const IntArr& piv, const Arr<S>& B, const std::string& precision, const std::string& backend) {
        const Precision p = prec(precision);
        const Backend b = back(backend);
        const S* lu = LU.data();
        const int* pv = piv.data();
        return solver_entry<S, Writes::Rhs, false, false>(LU, &B, &piv, [&](const Stack& s, S* x, int*, int*) {
          tsdx::lu_solve<S>(p, lu, pv, s.n, s.batch, x, s.nrhs, b);
        });
      },
      py::arg("LU"), py::arg("piv"), py::arg("B"), py::arg("precision") = "fp32", py::arg("backend") = "auto");
  m.def(
      name("round_to").c_str(),
      [=](const Arr<S>& x, const std::string& precision) {
        Arr<S> out = fresh_copy<S>(x);
        tsdx::round_to<S>(prec(precision), out.mutable_data(), out.size());
        return out;
      },
      py::arg("x"), py::arg("precision"));

  // fused factor + solve on the GPU, A untouched: (x, info)
  for (const bool spd : {true, false}) {
    m.def(
        name(spd ? "posv_cuda" : "gesv_cuda").c_str(),
        [spd](const Arr<S>& A, const Arr<S>& B) {
          const S* a = A.data();
          int rc = 0;
          py::object res = solver_entry<S, Writes::Rhs, false, true>(A, &B, nullptr, [&](const Stack& s, S* x, int*, int* info) {
            if (s.n < tsdx::kMinN || s.n > tsdx::kMaxN) {
              rc = TSDX_ERR_N;
              return;
            }
            if constexpr (std::is_same<S, double>::value)
              rc = spd ? tsdx_cuda_posv_solve_host_f64(a, s.n, s.batch, x, s.nrhs, info)
                       : tsdx_cuda_gesv_solve_host_f64(a, s.n, s.batch, x, s.nrhs, info);
            else
              rc = spd ? tsdx_cuda_posv_solve_host_f32(a, s.n, s.batch, x, s.nrhs, info)
                       : tsdx_cuda_gesv_solve_host_f32(a, s.n, s.batch, x, s.nrhs, info);
          });
          if (rc == TSDX_ERR_N)
            throw std::invalid_argument("matrix size n=" + std::to_string(A.shape(1)) + " outside supported range [1, 64]");
          tsdx::detail::check_cuda(rc);
          return res;
        },
        py::arg("A"), py::arg("B"));
  }
}

// ------------------------------------------------------------ metrics (float64)
using F64 = Arr<double>;

// solve metrics: f(A, x, b) per matrix
struct VectorMetric {
  const char* name;
  void (*fn)(const double*, const double*, const double*, int, std::int64_t, double*);
};
const VectorMetric kVectorMetrics[] = {{"solve_backward_error", &tsdx::solve_backward_error},
                                       {"solve_forward_error", &tsdx::solve_forward_error}};

py::array_t<double> per_matrix(py::ssize_t batch) { return py::array_t<double>(std::vector<py::ssize_t>{batch}); }

void bind_metrics(py::module_& m) {
  for (const VectorMetric& e : kVectorMetrics) {
    m.def(e.name, [fn = e.fn](const F64& A, const F64& x, const F64& b) {
      expect_vector(A, x, "x");
      expect_vector(A, b, "b");
      py::array_t<double> out = per_matrix(A.shape(0));
      fn(A.data(), x.data(), b.data(), static_cast<int>(A.shape(1)), A.shape(0), out.mutable_data());
      return out;
    });
  }
  // factorization metrics: the factor must hold as many elements as A
  m.def("chol_backward_error", [](const F64& A, const F64& L) {
    if (A.ndim() != 3 || A.shape(1) != A.shape(2) || L.ndim() != 3 || L.size() != A.size())
      throw std::invalid_argument("shape mismatch");
    py::array_t<double> out = per_matrix(A.shape(0));
    tsdx::chol_backward_error(A.data(), L.data(), static_cast<int>(A.shape(1)), A.shape(0), out.mutable_data());
    return out;
  });
  m.def("lu_backward_error", [](const F64& A, const F64& LU, const IntArr& piv) {
    if (A.ndim() != 3 || A.shape(1) != A.shape(2) || LU.size() != A.size() || piv.size() != A.shape(0) * A.shape(1))
      throw std::invalid_argument("shape mismatch");
    py::array_t<double> out = per_matrix(A.shape(0));
    tsdx::lu_backward_error(A.data(), LU.data(), piv.data(), static_cast<int>(A.shape(1)), A.shape(0), out.mutable_data());
    return out;
  });
  m.def("reference_solve", [](const F64& A, const F64& b) {
    expect_vector(A, b, "b");
    F64 x(std::vector<py::ssize_t>(b.shape(), b.shape() + b.ndim()));
    tsdx::reference_solve(A.data(), b.data(), static_cast<int>(A.shape(1)), A.shape(0), x.mutable_data());
    return x;
  });
}

}  // namespace

PYBIND11_MODULE(_core, m) {
  m.doc() = "B200-native batched small-matrix Cholesky/LU (drop-in for TinySolverDx _core)";
  bind_solvers<float>(m, "f32");
  bind_solvers<double>(m, "f64");
  m.def("has_cuda", &tsdx::has_cuda);
  m.def("has_openmp", &tsdx::has_openmp);
  m.def("num_threads", &tsdx::num_threads);
  m.def("set_num_threads", &tsdx::set_num_threads);
  m.def("unit_roundoff", [](const std::string& p) { return tsdx::unit_roundoff(option(kPrecision, p, "precision")); });
  bind_metrics(m);
}
