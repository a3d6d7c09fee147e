// tcon: pairwise tensor contraction with the label convention of the
// reference's ``tcon`` (src/utility/wrapper.jl:15-23, OMEinsum EinCode):
// positive labels are summed over, negative labels -1, -2, ... give the
// output order.  Planned as transpose-transpose-GEMM-transpose on
// column-major tensors:
//   * free labels of each operand are ordered as they appear in the output;
//   * the summed-label order is taken from A or from B, whichever needs fewer
//     permuted elements;
//   * an operand already laid out as [free, summed] or [summed, free] enters
//     the GEMM directly as op N / op T (no copy);
//   * the product is formed as [freeA, freeB] or, when the output lists all
//     of B's labels first, as its transpose [freeB, freeA]; only an
//     interleaved output needs a final permute.
#include "ctx.cuh"

#include <algorithm>
#include <map>

namespace ipeps {
namespace {

struct Plan {
  bool swap = false;  // compute with roles (A,B) swapped
  std::vector<int> fa, fb, kk;  // label lists
};

// position of each label in a label list
int find(const std::vector<int>& l, int x) {
  for (size_t i = 0; i < l.size(); ++i)
    if (l[i] == x) return int(i);
  return -1;
}

// Is tensor with labels `have` already ordered as concat(first, second)?
bool ordered_as(const std::vector<int>& have, const std::vector<int>& first, const std::vector<int>& second) {
  if (have.size() != first.size() + second.size()) return false;
  for (size_t i = 0; i < first.size(); ++i)
    if (have[i] != first[i]) return false;
  for (size_t i = 0; i < second.size(); ++i)
    if (have[first.size() + i] != second[i]) return false;
  return true;
}

// Unit-extent labels may be placed anywhere; drop them for ordering checks.
std::vector<int> strip_units(const std::vector<int>& labels, const std::map<int, int64_t>& ext) {
  std::vector<int> r;
  for (int l : labels)
    if (ext.at(l) != 1) r.push_back(l);
  return r;
}

struct Operand {
  Tensor t;     // possibly permuted copy
  char op;      // 'N' or 'T'
  int64_t ld;
};

// Bring X (labels lx) into a GEMM operand whose logical matrix is
// [rows, cols] where rows/cols are label lists.
Operand prepare(Ctx& c, const Tensor& X, const std::vector<int>& lx, const std::vector<int>& rows,
                const std::vector<int>& cols, const std::map<int, int64_t>& ext) {
  int64_t nr = 1, nc = 1;
  for (int l : rows) nr *= ext.at(l);
  for (int l : cols) nc *= ext.at(l);
  auto sx = strip_units(lx, ext), sr = strip_units(rows, ext), scl = strip_units(cols, ext);
  if (ordered_as(sx, sr, scl)) return {X, 'N', std::max<int64_t>(nr, 1)};
  if (ordered_as(sx, scl, sr)) return {X, 'T', std::max<int64_t>(nc, 1)};
  std::vector<int> perm;
  for (int l : rows) perm.push_back(find(lx, l));
  for (int l : cols) perm.push_back(find(lx, l));
  return {permute(c, X, perm), 'N', std::max<int64_t>(nr, 1)};
}

int64_t permute_cost(const std::vector<int>& lx, const std::vector<int>& r, const std::vector<int>& col,
                     const std::map<int, int64_t>& ext, int64_t numel) {
  auto sx = strip_units(lx, ext), sr = strip_units(r, ext), sc = strip_units(col, ext);
  if (ordered_as(sx, sr, sc) || ordered_as(sx, sc, sr)) return 0;
  return numel;
}

void contract(Ctx& c, const Tensor& A, const std::vector<int>& la, const Tensor& B,
              const std::vector<int>& lb, Tensor* out, bool accumulate) {
  IPEPS_CHECK(int(la.size()) == A.nd, "tcon: label count != rank of A " + shape_str(A));
  IPEPS_CHECK(int(lb.size()) == B.nd, "tcon: label count != rank of B " + shape_str(B));
  std::map<int, int64_t> ext;
  for (int i = 0; i < A.nd; ++i) ext[la[i]] = A.dims[i];
  for (int i = 0; i < B.nd; ++i) {
    auto it = ext.find(lb[i]);
    if (it != ext.end()) {
      IPEPS_CHECK(lb[i] > 0, "tcon: output label repeated");
      IPEPS_CHECK(it->second == B.dims[i], "tcon: extent mismatch on label " + std::to_string(lb[i]) +
                                               " A" + shape_str(A) + " B" + shape_str(B));
    } else {
      ext[lb[i]] = B.dims[i];
    }
  }
  std::vector<int> fa, fb, kA, kB;
  for (int l : la) (l < 0 ? fa : kA).push_back(l);
  for (int l : lb) (l < 0 ? fb : kB).push_back(l);
  IPEPS_CHECK(kA.size() == kB.size(), "tcon: summed labels must appear in both operands");
  for (int l : kA) IPEPS_CHECK(find(kB, l) >= 0, "tcon: label " + std::to_string(l) + " only in A");
  auto by_out = [](std::vector<int>& v) { std::sort(v.begin(), v.end(), [](int x, int y) { return x > y; }); };
  by_out(fa);
  by_out(fb);
  const int nout = int(fa.size() + fb.size());
  std::vector<int64_t> odims(nout);
  for (int i = 0; i < nout; ++i) {
    auto it = ext.find(-(i + 1));
    IPEPS_CHECK(it != ext.end(), "tcon: output labels must be -1..-n");
    odims[i] = it->second;
  }
  // output arrangement
  auto pos = [](int l) { return -l - 1; };
  int maxa = -1, mina = 1 << 30, maxb = -1, minb = 1 << 30;
  for (int l : fa) { maxa = std::max(maxa, pos(l)); mina = std::min(mina, pos(l)); }
  for (int l : fb) { maxb = std::max(maxb, pos(l)); minb = std::min(minb, pos(l)); }
  bool direct = fb.empty() || fa.empty() || maxa < minb;
  bool swapped = !direct && maxb < mina;
  // summed-label order: from A or from B
  int64_t costA = permute_cost(la, fa, kA, ext, A.numel()) + permute_cost(lb, kA, fb, ext, B.numel());
  int64_t costB = permute_cost(la, fa, kB, ext, A.numel()) + permute_cost(lb, kB, fb, ext, B.numel());
  const std::vector<int>& kk = (costB < costA) ? kB : kA;

  int64_t m = 1, n = 1, k = 1;
  for (int l : fa) m *= ext[l];
  for (int l : fb) n *= ext[l];
  for (int l : kk) k *= ext[l];

  DType dt = (A.dt == DType::C128 || B.dt == DType::C128) ? DType::C128 : DType::F64;
  Tensor Ac = A, Bc = B;
  if (A.dt != dt) Ac = to_complex(c, A);
  if (B.dt != dt) Bc = to_complex(c, B);

  Tensor res;
  bool need_final_perm = !(direct || swapped);
  if (accumulate) {
    IPEPS_CHECK(out && !out->empty() && out->numel() == m * n && out->dt == dt, "tcon_acc: bad output");
  }
  if (!need_final_perm && accumulate) res = *out;
  else if (!need_final_perm && out && !out->empty() && out->dt == dt && out->numel() == m * n) res = *out;
  else res = c.alloc(dt, direct || swapped ? odims : std::vector<int64_t>{m, n});

  if (k == 0 || m * n == 0) {
    if (!accumulate) IPEPS_CUDA(cudaMemsetAsync(res.data(), 0, res.bytes(), c.stream));
  } else if (!swapped) {
    Operand oa = prepare(c, Ac, la, fa, kk, ext);
    Operand ob = prepare(c, Bc, lb, kk, fb, ext);
    gemm(c, dt, oa.op, ob.op, m, n, k, cplx(1), oa.t.data(), oa.ld, ob.t.data(), ob.ld,
         cplx(accumulate && !need_final_perm ? 1.0 : 0.0), res.data(), m);
  } else {
    // C^T = B^T A^T : rows = fb, cols = fa
    Operand ob = prepare(c, Bc, lb, fb, kk, ext);
    Operand oa = prepare(c, Ac, la, kk, fa, ext);
    gemm(c, dt, ob.op, oa.op, n, m, k, cplx(1), ob.t.data(), ob.ld, oa.t.data(), oa.ld,
         cplx(accumulate ? 1.0 : 0.0), res.data(), n);
  }
  if (need_final_perm) {
    // res is [fa..., fb...] -> output order
    std::vector<int> cur(fa);
    cur.insert(cur.end(), fb.begin(), fb.end());
    std::vector<int64_t> cd;
    for (int l : cur) cd.push_back(ext[l]);
    Tensor r2 = res.reshape(cd);
    std::vector<int> perm(nout);
    for (int i = 0; i < nout; ++i) perm[i] = find(cur, -(i + 1));
    Tensor p = permute(c, r2, perm);
    if (accumulate) axpy(c, cplx(1), p, *out);
    else *out = p;
    return;
  }
  if (!accumulate) {
    res = res.reshape(odims);
    *out = res;
  }
}

}  // namespace

Tensor tcon(Ctx& c, const Tensor& A, const std::vector<int>& la, const Tensor& B,
            const std::vector<int>& lb) {
  Tensor out;
  contract(c, A, la, B, lb, &out, false);
  return out;
}

void tcon_acc(Ctx& c, Tensor& out, const Tensor& A, const std::vector<int>& la, const Tensor& B,
              const std::vector<int>& lb) {
  contract(c, A, la, B, lb, &out, true);
}

Tensor matmul(Ctx& c, const Tensor& A, char opA, const Tensor& B, char opB) {
  IPEPS_CHECK(A.nd == 2 && B.nd == 2, "matmul: 2-D operands expected");
  int64_t m = (opA == 'N') ? A.dims[0] : A.dims[1];
  int64_t ka = (opA == 'N') ? A.dims[1] : A.dims[0];
  int64_t kb = (opB == 'N') ? B.dims[0] : B.dims[1];
  int64_t n = (opB == 'N') ? B.dims[1] : B.dims[0];
  IPEPS_CHECK(ka == kb, "matmul: inner dimension mismatch " + shape_str(A) + " " + shape_str(B));
  DType dt = (A.dt == DType::C128 || B.dt == DType::C128) ? DType::C128 : DType::F64;
  Tensor Ac = A.dt == dt ? A : to_complex(c, A);
  Tensor Bc = B.dt == dt ? B : to_complex(c, B);
  Tensor C = c.alloc(dt, {m, n});
  gemm(c, dt, opA, opB, m, n, ka, cplx(1), Ac.data(), std::max<int64_t>(Ac.dims[0], 1), Bc.data(),
       std::max<int64_t>(Bc.dims[0], 1), cplx(0), C.data(), std::max<int64_t>(m, 1));
  return C;
}

void gemm(Ctx& c, DType dt, char opA, char opB, int64_t m, int64_t n, int64_t k,
          cuDoubleComplex alpha, const void* A, int64_t lda, const void* B, int64_t ldb,
          cuDoubleComplex beta, void* C, int64_t ldc, bool force_fp64) {
  if (dt == DType::F64 && c.precision == kPrecMixed && !force_fp64 && alpha.y == 0 && beta.y == 0 &&
      opA != 'C' && opB != 'C') {
    gemm_tf32x3(c, opA, opB, m, n, k, alpha.x, static_cast<const double*>(A), lda,
                static_cast<const double*>(B), ldb, beta.x, static_cast<double*>(C), ldc);
    return;
  }
  gemm_f64(c, dt, opA, opB, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc);
}

}  // namespace ipeps
