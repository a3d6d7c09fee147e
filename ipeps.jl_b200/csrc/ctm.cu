// CTMRG engine: nested-tensor algebra, the four directional moves, the
// energy and run_ctm.  Contraction labels follow the reference verbatim
// (file:line cited per function) so that every fused leg order is identical;
// only the renormalisation of the edge tensor (proj_*) uses a cheaper
// contraction order than the reference (same result, see proj_edge).
#include "ctm.cuh"
#include "linalg.cuh"

#include <chrono>
#include <cmath>

namespace ipeps {

// ------------------------------------------------------------ nested algebra
namespace {

void add_into(Ctx& c, Tensor& acc, const Tensor& t) {
  if (t.empty()) return;
  if (acc.empty()) {
    acc = t;
    return;
  }
  if (acc.dt != t.dt) {
    if (acc.dt == DType::F64) acc = to_complex(c, acc);
    else {
      axpy(c, cplx(1), t, acc);  // real into complex handled by axpy_rc
      return;
    }
  }
  axpy(c, cplx(1), t, acc);
}

}  // namespace

// nested_tensor.jl:77-92 (product rule), emptyT.jl:24-26 (EmptyT absorbs)
NT ntcon(Ctx& c, const NT& A, const std::vector<int>& la, const NT& B, const std::vector<int>& lb) {
  if (!A.nested && !B.nested) return NT(tcon(c, A.c[0], la, B.c[0], lb));
  NT r;
  r.nested = true;
  if (A.nested && B.nested) {
    static const int pairs[4][4][2] = {{{0, 0}, {-1, -1}, {-1, -1}, {-1, -1}},
                                       {{0, 1}, {1, 0}, {-1, -1}, {-1, -1}},
                                       {{0, 2}, {2, 0}, {-1, -1}, {-1, -1}},
                                       {{0, 3}, {3, 0}, {1, 2}, {2, 1}}};
    for (int o = 0; o < 4; ++o)
      for (int p = 0; p < 4; ++p) {
        int i = pairs[o][p][0], j = pairs[o][p][1];
        if (i < 0 || !A.has(i) || !B.has(j)) continue;
        add_into(c, r.c[o], tcon(c, A.c[i], la, B.c[j], lb));
      }
  } else if (A.nested) {
    for (int i = 0; i < 4; ++i)
      if (A.has(i)) r.c[i] = tcon(c, A.c[i], la, B.c[0], lb);
  } else {
    for (int i = 0; i < 4; ++i)
      if (B.has(i)) r.c[i] = tcon(c, A.c[0], la, B.c[i], lb);
  }
  return r;
}

NT nreshape(const NT& A, const std::vector<int64_t>& s) {
  NT r = A;
  for (int i = 0; i < 4; ++i)
    if (A.has(i)) r.c[i] = A.c[i].reshape(s);
  return r;
}

NT npermute(Ctx& c, const NT& A, const std::vector<int>& perm) {
  NT r = A;
  for (int i = 0; i < 4; ++i)
    if (A.has(i)) r.c[i] = permute(c, A.c[i], perm);
  return r;
}

// nested_tensor.jl:43-44 (componentwise product with a plain matrix)
NT nmatmul(Ctx& c, const NT& A, char opA, const NT& B, char opB) {
  IPEPS_CHECK(!(A.nested && B.nested), "nmatmul: nested x nested");
  NT r;
  r.nested = A.nested || B.nested;
  if (A.nested) {
    for (int i = 0; i < 4; ++i)
      if (A.has(i)) r.c[i] = matmul(c, A.c[i], opA, B.c[0], opB);
  } else if (B.nested) {
    for (int i = 0; i < 4; ++i)
      if (B.has(i)) r.c[i] = matmul(c, A.c[0], opA, B.c[i], opB);
  } else {
    r.c[0] = matmul(c, A.c[0], opA, B.c[0], opB);
  }
  return r;
}

// nested_tensor.jl:65: [A1, A2 e^{i phi}, A3 e^{-i phi}, A4]
NT nshift(Ctx& c, const NT& A, double phi) {
  if (!A.nested) return A;
  NT r = A;
  const double cs = std::cos(phi), sn = std::sin(phi);
  if (A.has(1)) {
    r.c[1] = clone(c, to_complex(c, A.c[1]));
    scale(c, r.c[1], cplx(cs, sn));
  }
  if (A.has(2)) {
    r.c[2] = clone(c, to_complex(c, A.c[2]));
    scale(c, r.c[2], cplx(cs, -sn));
  }
  return r;
}

// wrapper.jl:57 / nested_tensor.jl:70-75: divide by max|component 1|
void nrenormalize(Ctx& c, NT& A) {
  double* d_m = reinterpret_cast<double*>(c.scal->p) + 16;
  maxabs(c, A.c[0], d_m);
  for (int i = 0; i < 4; ++i)
    if (A.has(i)) {
      A.c[i] = A.c[i].buf.use_count() > 1 ? clone(c, A.c[i]) : A.c[i];
      scale_inv(c, A.c[i], d_m);
    }
}

// ------------------------------------------------------------ environment
NT Env::all_A() const {  // ctm_tensor.jl:20-27
  if (!nested) return NT(A);
  NT r;
  r.nested = true;
  r.c[0] = A;
  r.c[1] = B;
  return r;
}
NT Env::all_Ad() const {  // ctm_tensor.jl:29-36
  if (!nested) return NT(Ad);
  NT r;
  r.nested = true;
  r.c[0] = Ad;
  r.c[2] = Bd;
  return r;
}
NT Env::all_C(int i) const {  // ctm_tensor.jl:38-45
  if (!nested) return NT(Cs[i]);
  NT r;
  r.nested = true;
  r.c = {Cs[i], B_Cs[i], Bd_Cs[i], BB_Cs[i]};
  return r;
}
NT Env::all_E(int i) const {  // ctm_tensor.jl:47-55
  if (!nested) return NT(Es[i]);
  NT r;
  r.nested = true;
  r.c = {Es[i], B_Es[i], Bd_Es[i], BB_Es[i]};
  return r;
}

// ctm_tensor.jl:97-130
void init_ctm1(Env& e) {
  Ctx& c = *e.ctx;
  const int64_t D = e.D, D2 = int64_t(D) * D;
  auto mk = [&](const std::vector<int>& la, const std::vector<int>& lb, std::vector<int64_t> shape) {
    NT t(tcon(c, e.A, la, e.Ad, lb).reshape(shape));
    nrenormalize(c, t);
    return t.c[0];
  };
  e.Cs[0] = mk({1, 2, -1, -3, 3}, {1, 2, -2, -4, 3}, {D2, D2});
  e.Cs[1] = mk({1, -1, -3, 2, 3}, {1, -2, -4, 2, 3}, {D2, D2});
  e.Cs[2] = mk({-1, -3, 1, 2, 3}, {-2, -4, 1, 2, 3}, {D2, D2});
  e.Cs[3] = mk({-1, 1, 2, -3, 3}, {-2, 1, 2, -4, 3}, {D2, D2});
  e.Es[0] = mk({1, -1, -5, -3, 2}, {1, -2, -6, -4, 2}, {D2, D2, D, D});
  e.Es[1] = mk({-1, -5, -3, 1, 2}, {-2, -6, -4, 1, 2}, {D2, D2, D, D});
  e.Es[2] = mk({-5, -1, 1, -3, 2}, {-6, -2, 1, -4, 2}, {D2, D2, D, D});
  e.Es[3] = mk({-1, 1, -3, -5, 2}, {-2, 1, -4, -6, 2}, {D2, D2, D, D});
  for (int i = 0; i < 4; ++i) e.cache[i].V = Tensor();
}

// ------------------------------------------------------------ projectors
namespace {

int64_t prod3(const Tensor& t) { return t.dims[0] * t.dims[1] * t.dims[2]; }

// ctmrg.jl:122-153
void quarters_left(Ctx& c, Env& e, MatRef& R1, MatRef& R2) {
  const Tensor &C1 = e.Cs[0], &C4 = e.Cs[3], &E1 = e.Es[0], &E3 = e.Es[2], &E4 = e.Es[3];
  const Tensor &A = e.A, &Ad = e.Ad;
  Tensor C1E1 = tcon(c, C1, {-1, 1}, E1, {1, -2, -3, -4});
  Tensor CEE4 = tcon(c, C1E1, {1, -2, -5, -3}, E4, {1, -1, -6, -4});
  Tensor CEEA = tcon(c, CEE4, {-1, -2, -3, -4, 1, 2}, A, {1, 2, -5, -6, -7});
  Tensor LU = tcon(c, CEEA, {-1, -4, 1, 2, -2, -5, 3}, Ad, {1, 2, -3, -6, 3});
  R1 = MatRef{LU.reshape({prod3(LU), -1}), true};
  Tensor C4E3 = tcon(c, C4, {-1, 1}, E3, {1, -2, -3, -4});
  Tensor CEE4b = tcon(c, C4E3, {1, -2, -6, -4}, E4, {-1, 1, -5, -3});
  Tensor CEEAb = tcon(c, CEE4b, {-1, -2, -3, -4, 1, 2}, A, {-5, 1, 2, -6, -7});
  Tensor LB = tcon(c, CEEAb, {-1, -4, 1, 2, -2, -5, 3}, Ad, {-3, 1, 2, -6, 3});
  R2 = MatRef{LB.reshape({prod3(LB), -1}), false};
}

// ctmrg.jl:155-186
void quarters_right(Ctx& c, Env& e, MatRef& R1, MatRef& R2) {
  const Tensor &C2 = e.Cs[1], &C3 = e.Cs[2], &E1 = e.Es[0], &E2 = e.Es[1], &E3 = e.Es[2];
  const Tensor &A = e.A, &Ad = e.Ad;
  Tensor C2E1 = tcon(c, C2, {1, -2}, E1, {-1, 1, -3, -4});
  Tensor CEE2 = tcon(c, C2E1, {-1, 1, -5, -3}, E2, {1, -2, -6, -4});
  Tensor CEEA = tcon(c, CEE2, {-1, -2, -3, -4, 1, 2}, A, {1, -5, -6, 2, -7});
  Tensor RU = tcon(c, CEEA, {-1, -4, 1, 2, -2, -5, 3}, Ad, {1, -3, -6, 2, 3});
  R1 = MatRef{RU.reshape({prod3(RU), -1}), false};
  Tensor C3E3 = tcon(c, C3, {-1, 1}, E3, {-2, 1, -3, -4});
  Tensor CEE2b = tcon(c, C3E3, {1, -2, -5, -3}, E2, {-1, 1, -6, -4});
  Tensor CEEAb = tcon(c, CEE2b, {-1, -2, -5, -6, 1, 2}, A, {-3, -4, 1, 2, -7});
  Tensor RB = tcon(c, CEEAb, {-1, -4, -2, -5, 1, 2, 3}, Ad, {-3, -6, 1, 2, 3});
  R2 = MatRef{RB.reshape({prod3(RB), -1}), false};
}

// ctmrg.jl:188-219
void quarters_top(Ctx& c, Env& e, MatRef& R1, MatRef& R2) {
  const Tensor &C1 = e.Cs[0], &C2 = e.Cs[1], &E1 = e.Es[0], &E2 = e.Es[1], &E4 = e.Es[3];
  const Tensor &A = e.A, &Ad = e.Ad;
  Tensor C1E4 = tcon(c, C1, {1, -2}, E4, {1, -1, -3, -4});
  Tensor CEE1 = tcon(c, C1E4, {-1, 1, -6, -4}, E1, {1, -2, -5, -3});
  Tensor CEEA = tcon(c, CEE1, {-1, -2, -5, -6, 1, 2}, A, {1, 2, -3, -4, -7});
  Tensor UL = tcon(c, CEEA, {-1, -4, -2, -5, 1, 2, 3}, Ad, {1, 2, -3, -6, 3});
  R1 = MatRef{UL.reshape({prod3(UL), -1}), false};
  Tensor C2E2 = tcon(c, C2, {-1, 1}, E2, {1, -2, -3, -4});
  Tensor CEE1b = tcon(c, C2E2, {1, -2, -6, -4}, E1, {-1, 1, -5, -3});
  Tensor CEEAb = tcon(c, CEE1b, {-1, -2, -5, -6, 1, 2}, A, {1, -3, -4, 2, -7});
  Tensor UR = tcon(c, CEEAb, {-1, -4, -2, -5, 1, 2, 3}, Ad, {1, -3, -6, 2, 3});
  R2 = MatRef{UR.reshape({prod3(UR), -1}), false};
}

// ctmrg.jl:221-252
void quarters_bottom(Ctx& c, Env& e, MatRef& R1, MatRef& R2) {
  const Tensor &C3 = e.Cs[2], &C4 = e.Cs[3], &E2 = e.Es[1], &E3 = e.Es[2], &E4 = e.Es[3];
  const Tensor &A = e.A, &Ad = e.Ad;
  Tensor C4E4 = tcon(c, C4, {1, -2}, E4, {-1, 1, -3, -4});
  Tensor CEE3 = tcon(c, C4E4, {-1, 1, -5, -3}, E3, {1, -2, -6, -4});
  Tensor CEEA = tcon(c, CEE3, {-1, -2, -5, -6, 1, 2}, A, {-3, 1, 2, -4, -7});
  Tensor BL = tcon(c, CEEA, {-1, -4, -2, -5, 1, 2, 3}, Ad, {-3, 1, 2, -6, 3});
  R1 = MatRef{BL.reshape({prod3(BL), -1}), false};
  Tensor C3E2 = tcon(c, C3, {1, -2}, E2, {-1, 1, -3, -4});
  Tensor CEE3b = tcon(c, C3E2, {-1, 1, -6, -4}, E3, {-2, 1, -5, -3});
  Tensor CEEAb = tcon(c, CEE3b, {-1, -2, -5, -6, 1, 2}, A, {-3, -4, 1, 2, -7});
  Tensor BR = tcon(c, CEEAb, {-1, -4, -2, -5, 1, 2, 3}, Ad, {-3, -6, 1, 2, 3});
  R2 = MatRef{BR.reshape({prod3(BR), -1}), true};
}

// New edge tensor of a move.  The reference (ctmrg.jl:284-290 and the right,
// top and bottom analogues) forms T*A*A' (chi^2 D^6 elements) and then
// contracts Pd and P (2 chi^3 D^6 flops).  The same tensor
//   newE[c,c2,o,o'] = sum Pd[c,(a,g,g')] E[a,b,k,k'] A[..g..k..h..o..s] A'[..g'..k'..h'..o'..s] P[(b,h,h'),c2]
// is contracted here as ((Pd*E)*A)*A' then *P, which costs
// 4 chi^3 D^4 + 4 chi^2 D^6 d flops and never materialises chi^2 D^6.
// Legs of A are (up, left, down, right, phys) = 0..4; lg/le/lh/lo are the
// legs grouped with Pd, contracted with E, grouped with P, and left open.
NT proj_edge(Ctx& c, const NT& E, const NT& A, const NT& Ad, const Tensor& P, const Tensor& Pd, int lg,
             int le, int lh, int lo) {
  const int64_t chiE = E.c[0].dims[0], D = A.c[0].dims[0];
  NT Pdr(Pd.reshape({Pd.dims[0], chiE, D, D}));
  NT X2 = ntcon(c, Pdr, {-1, 1, -2, -3}, E, {1, -4, -5, -6});  // (c, g, g', b, k, k')
  std::vector<int> la(5);
  la[lg] = 1;
  la[le] = 2;
  la[lh] = -5;
  la[lo] = -6;
  la[4] = -7;
  NT X3 = ntcon(c, X2, {-1, 1, -2, -3, 2, -4}, A, la);  // (c, g', b, k', h, o, s)
  std::vector<int> lad(5);
  lad[lg] = 1;
  lad[le] = 2;
  lad[lh] = -5;
  lad[lo] = -6;
  lad[4] = 3;
  NT X4 = ntcon(c, X3, {-1, 1, -2, 2, -3, -4, 3}, Ad, lad);  // (c, b, h, o, h', o')
  const int64_t chiB = E.c[0].dims[1];
  NT Pr(P.reshape({chiB, D, D, P.dims[1]}));
  return ntcon(c, X4, {-1, 1, 2, -3, 3, -4}, Pr, {1, 2, 3, -2});  // (c, c2, o, o')
}

}  // namespace

// One directional move: *_rg (ctmrg.jl:66-120) = projector + proj_* +
// renormalize + up_*.
std::vector<double> ctm_move(Env& e, int dir) {
  Ctx& c = *e.ctx;
  IPEPS_CHECK(e.dt == DType::F64, "ctm_move: complex A needs the complex projector (not built)");
  auto t0 = std::chrono::steady_clock::now();
  MatRef R1, R2;
  switch (dir) {
    case 0: quarters_left(c, e, R1, R2); break;
    case 1: quarters_right(c, e, R1, R2); break;
    case 2: quarters_top(c, e, R1, R2); break;
    default: quarters_bottom(c, e, R1, R2); break;
  }
  ProjResult pr = get_projector(c, R1, R2, e.prm.chi, e.prm.svd, &e.cache[dir]);
  R1 = MatRef();
  R2 = MatRef();
  const Tensor& P = pr.P1;
  const Tensor& Pd = pr.P2;
  NT A = e.all_A(), Ad = e.all_Ad();
  NT nC_a, nE, nC_b;
  if (dir == 0) {  // proj_left ctmrg.jl:267-293
    NT C1 = e.all_C(0), C4 = e.all_C(3), E1 = e.all_E(0), E3 = e.all_E(2), E4 = e.all_E(3);
    NT C1E1 = ntcon(c, C1, {-2, 1}, E1, {1, -1, -3, -4});
    nC_a = npermute(c, nmatmul(c, nreshape(C1E1, {C1E1.c[0].dims[0], -1}), 'N', NT(P), 'N'), {1, 0});
    NT C4E3 = ntcon(c, C4, {-1, 1}, E3, {1, -4, -2, -3});
    nC_b = nmatmul(c, NT(Pd), 'N', nreshape(C4E3, {-1, C4E3.c[0].dims[3]}), 'N');
    nE = proj_edge(c, E4, A, Ad, P, Pd, 0, 1, 2, 3);
  } else if (dir == 1) {  // proj_right ctmrg.jl:295-320
    NT C2 = e.all_C(1), C3 = e.all_C(2), E1 = e.all_E(0), E2 = e.all_E(1), E3 = e.all_E(2);
    NT C2E1 = ntcon(c, C2, {1, -2}, E1, {-1, 1, -3, -4});
    nC_a = nmatmul(c, nreshape(C2E1, {C2E1.c[0].dims[0], -1}), 'N', NT(P), 'N');
    NT C3E3 = ntcon(c, C3, {-1, 1}, E3, {-4, 1, -2, -3});
    nC_b = nmatmul(c, NT(Pd), 'N', nreshape(C3E3, {-1, C3E3.c[0].dims[3]}), 'N');
    nE = proj_edge(c, E2, A, Ad, P, Pd, 0, 3, 2, 1);
  } else if (dir == 2) {  // proj_top ctmrg.jl:322-347
    NT C1 = e.all_C(0), C2 = e.all_C(1), E1 = e.all_E(0), E2 = e.all_E(1), E4 = e.all_E(3);
    NT C1E4 = ntcon(c, C1, {1, -2}, E4, {1, -1, -3, -4});
    nC_a = nmatmul(c, nreshape(C1E4, {C1E4.c[0].dims[0], -1}), 'N', NT(P), 'N');
    NT C2E2 = ntcon(c, C2, {-1, 1}, E2, {1, -4, -2, -3});
    nC_b = nmatmul(c, NT(Pd), 'N', nreshape(C2E2, {-1, C2E2.c[0].dims[3]}), 'N');
    nE = proj_edge(c, E1, A, Ad, P, Pd, 1, 0, 3, 2);
  } else {  // proj_bottom ctmrg.jl:349-375
    NT C3 = e.all_C(2), C4 = e.all_C(3), E2 = e.all_E(1), E3 = e.all_E(2), E4 = e.all_E(3);
    NT C4E4 = ntcon(c, C4, {1, -2}, E4, {-1, 1, -3, -4});
    nC_a = nmatmul(c, nreshape(C4E4, {C4E4.c[0].dims[0], -1}), 'N', NT(P), 'N');
    NT C3E2 = ntcon(c, C3, {1, -1}, E2, {-4, 1, -2, -3});
    nC_b = npermute(c, nmatmul(c, NT(Pd), 'N', nreshape(C3E2, {-1, C3E2.c[0].dims[3]}), 'N'), {1, 0});
    nE = proj_edge(c, E3, A, Ad, P, Pd, 1, 2, 3, 0);
  }
  nrenormalize(c, nC_a);
  nrenormalize(c, nE);
  nrenormalize(c, nC_b);
  // up_* (ctmrg.jl:377-491): slots per direction
  int ia, ib, ie;
  double phi;
  switch (dir) {
    case 0: ia = 0; ib = 3; ie = 3; phi = -e.px; break;  // C1, C4, E4
    case 1: ia = 1; ib = 2; ie = 1; phi = e.px; break;   // C2, C3, E2
    case 2: ia = 0; ib = 1; ie = 0; phi = -e.py; break;  // C1, C2, E1
    default: ia = 3; ib = 2; ie = 2; phi = e.py; break;  // C4, C3, E3
  }
  if (e.nested) {
    nC_a = nshift(c, nC_a, phi);
    nC_b = nshift(c, nC_b, phi);
    nE = nshift(c, nE, phi);
    e.B_Cs[ia] = nC_a.c[1]; e.Bd_Cs[ia] = nC_a.c[2]; e.BB_Cs[ia] = nC_a.c[3];
    e.B_Cs[ib] = nC_b.c[1]; e.Bd_Cs[ib] = nC_b.c[2]; e.BB_Cs[ib] = nC_b.c[3];
    e.B_Es[ie] = nE.c[1]; e.Bd_Es[ie] = nE.c[2]; e.BB_Es[ie] = nE.c[3];
  }
  e.Cs[ia] = nC_a.c[0];
  e.Cs[ib] = nC_b.c[0];
  e.Es[ie] = nE.c[0];
  e.moves++;
  auto t1 = std::chrono::steady_clock::now();
  e.move_seconds += std::chrono::duration<double>(t1 - t0).count();
  return pr.s_host;
}

// ctmrg.jl:57-64
std::vector<double> rg_step(Env& e) {
  std::vector<double> s = ctm_move(e, 0);
  ctm_move(e, 1);
  ctm_move(e, 2);
  ctm_move(e, 3);
  e.last_s = s;
  return s;
}

// ------------------------------------------------------------ observables
namespace {

// evaluation.jl:169-200
NT get_dm_h(Ctx& c, const NT& C1, const NT& C2, const NT& C3, const NT& C4, const NT& E1l, const NT& E1r,
            const NT& E2, const NT& E3l, const NT& E3r, const NT& E4, const NT& Al, const NT& Ar, const NT& Adl,
            const NT& Adr) {
  NT C1E1 = ntcon(c, C1, {-1, 1}, E1l, {1, -2, -3, -4});
  NT LU = ntcon(c, C1E1, {-1, -2, -3, 1}, Adl, {1, -4, -5, -6, -7});
  NT C4E3 = ntcon(c, C4, {-1, 1}, E3l, {1, -2, -3, -4});
  NT CEE4 = ntcon(c, E4, {-1, 1, -3, -5}, C4E3, {1, -2, -4, -6});
  NT LB = ntcon(c, CEE4, {-1, -2, 1, 2, -4, -5}, Al, {-3, 1, 2, -6, -7});
  NT L = ntcon(c, LB, {1, -2, 2, 3, 4, -3, -5}, LU, {1, -1, 2, 3, 4, -4, -6});
  NT C2E1 = ntcon(c, C2, {1, -2}, E1r, {-1, 1, -3, -4});
  NT RU = ntcon(c, C2E1, {-1, -2, 1, -3}, Ar, {1, -4, -5, -6, -7});
  NT C3E3 = ntcon(c, C3, {-1, 1}, E3r, {-2, 1, -3, -4});
  NT CEE2 = ntcon(c, C3E3, {1, -2, -3, -5}, E2, {-1, 1, -4, -6});
  NT RB = ntcon(c, CEE2, {-1, -2, -3, -4, 1, 2}, Adr, {-5, -6, 1, 2, -7});
  NT R = ntcon(c, RU, {-1, 1, 2, -3, 3, 4, -5}, RB, {1, -2, 3, 4, 2, -4, -6});
  NT roh = ntcon(c, L, {1, 2, 3, 4, -1, -3}, R, {1, 2, 3, 4, -2, -4});
  const int64_t d = Al.c[0].dims[4];
  return nreshape(roh, {d * d, d * d});
}

// evaluation.jl:217-248
NT get_dm_v(Ctx& c, const NT& C1, const NT& C2, const NT& C3, const NT& C4, const NT& E1, const NT& E2u,
            const NT& E2d, const NT& E3, const NT& E4u, const NT& E4d, const NT& Au, const NT& Ad, const NT& Adu,
            const NT& Add) {
  NT C1E1 = ntcon(c, C1, {-1, 1}, E1, {1, -2, -3, -4});
  NT CEE4 = ntcon(c, C1E1, {1, -2, -3, -5}, E4u, {1, -1, -4, -6});
  NT UL = ntcon(c, CEE4, {-1, -2, 1, 2, -3, -4}, Au, {1, 2, -5, -6, -7});
  NT C2E2 = ntcon(c, C2, {-1, 1}, E2u, {1, -2, -3, -4});
  NT UR = ntcon(c, C2E2, {-1, -2, -3, 1}, Adu, {-4, -5, -6, 1, -7});
  NT U = ntcon(c, UL, {-1, 1, 3, 4, -3, 2, -5}, UR, {1, -2, 2, 3, 4, -4, -6});
  NT C4E3 = ntcon(c, C4, {-1, 1}, E3, {1, -2, -3, -4});
  NT CEE4b = ntcon(c, C4E3, {1, -2, -4, -6}, E4d, {-1, 1, -3, -5});
  NT BL = ntcon(c, CEE4b, {-1, -2, -3, -4, 1, 2}, Add, {-5, 1, 2, -6, -7});
  NT C3E2 = ntcon(c, C3, {1, -2}, E2d, {-1, 1, -3, -4});
  NT BR = ntcon(c, C3E2, {-1, -2, 1, -3}, Ad, {-4, -5, -6, 1, -7});
  NT B = ntcon(c, BL, {-1, 1, 2, 3, -4, 4, -6}, BR, {-2, 1, 4, -3, 2, 3, -5});
  NT rov = ntcon(c, U, {1, 2, 3, 4, -1, -3}, B, {1, 2, 3, 4, -2, -4});
  const int64_t d = Au.c[0].dims[4];
  return nreshape(rov, {d * d, d * d});
}

// out[0..1] = tr(H rho) (complex), out[2..3] = tr(rho) (complex); FP64
__global__ void dm_trace_kernel(const double* rho, int rho_complex, const double2* H, int n, double* out) {
  // one warp
  double hr = 0, hi = 0, tr = 0, ti = 0;
  for (int t = threadIdx.x; t < n * n; t += 32) {
    int i = t % n, j = t / n;  // tr(H rho) = sum_ij H[i,j] rho[j,i]
    double rr, ri;
    int64_t idx = int64_t(j) + int64_t(i) * n;
    if (rho_complex) { rr = rho[2 * idx]; ri = rho[2 * idx + 1]; }
    else { rr = rho[idx]; ri = 0; }
    double2 h = H[i + int64_t(j) * n];
    hr += h.x * rr - h.y * ri;
    hi += h.x * ri + h.y * rr;
    if (i == j) { tr += rr; ti += ri; }
  }
  for (int o = 16; o; o >>= 1) {
    hr += __shfl_xor_sync(0xffffffffu, hr, o);
    hi += __shfl_xor_sync(0xffffffffu, hi, o);
    tr += __shfl_xor_sync(0xffffffffu, tr, o);
    ti += __shfl_xor_sync(0xffffffffu, ti, o);
  }
  if (threadIdx.x == 0) { out[0] = hr; out[1] = hi; out[2] = tr; out[3] = ti; }
}

struct Traces {
  std::complex<double> trH, tr;
};

// traces of several (rho, H) pairs in one host round trip
std::vector<Traces> dm_traces(Ctx& c, const std::vector<std::pair<Tensor, Tensor>>& items) {
  const int n = int(items.size());
  double* d_out = reinterpret_cast<double*>(c.scal->p) + 64;
  IPEPS_CHECK(n * 4 <= 256, "dm_traces: too many items");
  for (int i = 0; i < n; ++i) {
    const Tensor& rho = items[i].first;
    const Tensor& H = items[i].second;
    int d2 = int(rho.dims[0]);
    IPEPS_CHECK(H.dims[0] == d2 && H.dt == DType::C128, "dm_traces: H must be complex d^2 x d^2");
    dm_trace_kernel<<<1, 32, 0, c.stream>>>(rho.f64(), rho.dt == DType::C128, static_cast<const double2*>(H.data()),
                                            d2, d_out + 4 * i);
    IPEPS_LAUNCH_CHECK();
    c.count(KFam::Reduce);
  }
  std::vector<double> h(4 * n);
  IPEPS_CUDA(cudaMemcpyAsync(h.data(), d_out, h.size() * 8, cudaMemcpyDeviceToHost, c.stream));
  c.sync();
  std::vector<Traces> r(n);
  for (int i = 0; i < n; ++i) {
    r[i].trH = {h[4 * i], h[4 * i + 1]};
    r[i].tr = {h[4 * i + 2], h[4 * i + 3]};
  }
  return r;
}

}  // namespace

// evaluation.jl:15-29 with get_dms (only_gs) evaluation.jl:124-156
void gs_energy(Env& e, const Tensor& Hh, const Tensor& Hv, std::complex<double>* E, std::complex<double>* Na) {
  Ctx& c = *e.ctx;
  NT C1(e.Cs[0]), C2(e.Cs[1]), C3(e.Cs[2]), C4(e.Cs[3]);
  NT E1(e.Es[0]), E2(e.Es[1]), E3(e.Es[2]), E4(e.Es[3]);
  NT A(e.A), Ad(e.Ad);
  NT roh = get_dm_h(c, C1, C2, C3, C4, E1, E1, E2, E3, E3, E4, A, A, Ad, Ad);
  NT rov = get_dm_v(c, C1, C2, C3, C4, E1, E2, E2, E3, E4, E4, A, A, Ad, Ad);
  auto t = dm_traces(c, {{roh.c[0], Hh}, {rov.c[0], Hv}});
  const std::complex<double> Nh = t[0].tr, Nv = t[1].tr;
  *Na = (Nh + Nv) / 2.0;
  *E = t[0].trH / Nh + t[1].trH / Nv;
}

// evaluation.jl:31-45 (get_dms with only_gs = false)
double es_energy(Env& e, const Tensor& Hh, const Tensor& Hv) {
  Ctx& c = *e.ctx;
  IPEPS_CHECK(e.nested, "es_energy: no B set");
  NT C1 = e.all_C(0), C2 = e.all_C(1), C3 = e.all_C(2), C4 = e.all_C(3);
  NT E1 = e.all_E(0), E2 = e.all_E(1), E3 = e.all_E(2), E4 = e.all_E(3);
  NT A = e.all_A(), Ad = e.all_Ad();
  const double px = e.px, py = e.py;
  NT roh = get_dm_h(c, C1, nshift(c, C2, px), nshift(c, C3, px), C4, E1, nshift(c, E1, px), nshift(c, E2, px), E3,
                    nshift(c, E3, px), E4, A, nshift(c, A, px), Ad, nshift(c, Ad, px));
  NT rov = get_dm_v(c, C1, C2, nshift(c, C3, py), nshift(c, C4, py), E1, E2, nshift(c, E2, py), nshift(c, E3, py),
                    E4, nshift(c, E4, py), A, nshift(c, A, py), Ad, nshift(c, Ad, py));
  std::vector<std::pair<Tensor, Tensor>> items;
  std::vector<int> which;
  for (int i = 0; i < 4; ++i) {
    if (roh.has(i)) { items.push_back({roh.c[i], Hh}); which.push_back(i); }
  }
  for (int i = 0; i < 4; ++i) {
    if (rov.has(i)) { items.push_back({rov.c[i], Hv}); which.push_back(4 + i); }
  }
  auto t = dm_traces(c, items);
  std::complex<double> trHh[4] = {}, trHv[4] = {}, trh0 = 0, trv0 = 0;
  for (size_t i = 0; i < items.size(); ++i) {
    int w = which[i];
    if (w < 4) { trHh[w] = t[i].trH; if (w == 0) trh0 = t[i].tr; }
    else { trHv[w - 4] = t[i].trH; if (w == 4) trv0 = t[i].tr; }
  }
  const double Nh = trh0.real(), Nv = trv0.real();
  std::complex<double> E4v = trHh[3] / Nh + trHv[3] / Nv;
  return E4v.real();
}

// evaluation.jl:110-122
static NT get_single_dm(Ctx& c, const NT& C1, const NT& C2, const NT& C3, const NT& C4, const NT& E1, const NT& E2,
                        const NT& E3, const NT& E4) {
  NT C1E1 = ntcon(c, C1, {-1, 1}, E1, {1, -2, -3, -4});
  NT CEC2 = ntcon(c, C1E1, {-1, 1, -3, -4}, C2, {1, -2});
  NT CECE4 = ntcon(c, CEC2, {1, -2, -3, -5}, E4, {1, -1, -4, -6});
  NT C4E3 = ntcon(c, C4, {-1, 1}, E3, {1, -2, -3, -4});
  NT CEC3 = ntcon(c, C4E3, {-1, 1, -3, -4}, C3, {-2, 1});
  NT CECE2 = ntcon(c, CEC3, {-1, 1, -3, -5}, E2, {-2, 1, -4, -6});
  return ntcon(c, CECE4, {1, 2, -1, -2, -5, -6}, CECE2, {1, 2, -3, -4, -7, -8});
}

static std::complex<double> scalar_of(Ctx& c, const Tensor& t) {
  double h[2] = {0, 0};
  IPEPS_CUDA(cudaMemcpyAsync(h, t.data(), t.dt == DType::F64 ? 8 : 16, cudaMemcpyDeviceToHost, c.stream));
  c.sync();
  return {h[0], t.dt == DType::F64 ? 0.0 : h[1]};
}

// evaluation.jl:47-59
std::complex<double> gs_norm(Env& e) {
  Ctx& c = *e.ctx;
  NT n_dm = get_single_dm(c, e.Cs[0], e.Cs[1], e.Cs[2], e.Cs[3], e.Es[0], e.Es[1], e.Es[2], e.Es[3]);
  Tensor ndm_Ad = tcon(c, n_dm.c[0], {-1, -2, -3, -4, 1, 2, 3, 4}, e.Ad, {1, 2, 3, 4, -5});
  Tensor nrm0 = tcon(c, ndm_Ad, {1, 2, 3, 4, 5}, e.A, {1, 2, 3, 4, 5});
  return scalar_of(c, nrm0);
}

// evaluation.jl:61-77
std::complex<double> all_norm(Env& e, Tensor* envB) {
  Ctx& c = *e.ctx;
  IPEPS_CHECK(e.nested, "all_norm: no B set");
  NT n_dm = get_single_dm(c, e.all_C(0), e.all_C(1), e.all_C(2), e.all_C(3), e.all_E(0), e.all_E(1), e.all_E(2),
                          e.all_E(3));
  NT ndm_A = ntcon(c, n_dm, {1, 2, 3, 4, -1, -2, -3, -4}, e.all_A(), {1, 2, 3, 4, -5});
  NT all = ntcon(c, ndm_A, {1, 2, 3, 4, 5}, e.all_Ad(), {1, 2, 3, 4, 5});
  std::complex<double> n1 = scalar_of(c, all.c[0]);
  IPEPS_CHECK(ndm_A.has(1), "all_norm: empty B slot");
  if (envB) {
    *envB = clone(c, to_complex(c, ndm_A.c[1]));
    scale(c, *envB, cplx((1.0 / n1).real(), (1.0 / n1).imag()));
  }
  Tensor Nb = tcon(c, ndm_A.c[1], {1, 2, 3, 4, 5}, e.Bd, {1, 2, 3, 4, 5});
  return scalar_of(c, Nb) / n1;
}

// ctmrg.jl:1-55
int run_ctm(Env& e, int conv_mode, const Tensor* Hh, const Tensor* Hv, double* last_diff, bool* converged) {
  std::vector<double> diffs{1.0};
  std::complex<double> conv = 1.0;
  std::vector<double> conv_s{1.0};
  e.log.clear();
  int i = 1;
  bool done = false;
  for (; i <= e.prm.max_iter; ++i) {
    std::vector<double> s = rg_step(e);
    CtmLogEntry le{i, 0, 0, 0, int(s.size())};
    if (conv_mode == 0 || conv_mode == 2) {
      std::complex<double> old = conv;
      if (conv_mode == 0) {
        std::complex<double> E, Na;
        gs_energy(e, *Hh, *Hv, &E, &Na);
        conv = E;
      } else {
        double Ees = es_energy(e, *Hh, *Hv);
        conv = Ees / all_norm(e, nullptr);
      }
      diffs.push_back(std::abs(conv - old));
      le.obj_re = conv.real();
      le.obj_im = conv.imag();
    } else {
      std::vector<double> old = conv_s;
      conv_s = s;
      if (conv_s.size() == old.size()) {
        double acc = 0;
        for (size_t j = 0; j < s.size(); ++j) acc += (conv_s[j] - old[j]) * (conv_s[j] - old[j]);
        diffs.push_back(std::sqrt(acc));
      }
    }
    le.diff = diffs.back();
    e.log.push_back(le);
    if (i >= e.prm.min_iter && diffs.back() < e.prm.rg_tol) {
      done = true;
      break;
    }
  }
  if (last_diff) *last_diff = diffs.back();
  if (converged) *converged = done;
  return done ? i : e.prm.max_iter;
}

}  // namespace ipeps
