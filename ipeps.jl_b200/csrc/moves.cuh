// The contraction sequences of the directional CTMRG move and of the
// density matrices, written once and instantiated for a tensor "policy":
//   NTPolicy  - forward engine on plain or nested (4-component) tensors
//   ADPolicy  - the same sequence recorded on the reverse-mode tape
// A policy P provides: type T; tc(a, la, b, lb) (tcon); rs(a, shape)
// (Julia reshape); pm(a, perm) (permutedims, 0-based); mm(a, b) (matrix
// product a*b); dim(a, i).
// Labels are the reference's, verbatim; file:line per function.
#pragma once
#include <array>
#include <vector>

namespace ipeps {

template <class P>
struct QuarterPair {
  typename P::T R1, R2;  // N x N matrices (possibly as transposed views)
  bool t1 = false, t2 = false;
};

template <class P>
using Arr4 = std::array<typename P::T, 4>;

template <class P>
int64_t prod3(P& p, const typename P::T& x) {
  return p.dim(x, 0) * p.dim(x, 1) * p.dim(x, 2);
}

// get_projector_{left,right,top,bottom} without the SVD (ctmrg.jl:122-252).
// Projectors are built from the plain environment only (ctmrg.jl:122-134).
template <class P>
QuarterPair<P> quarters(P& p, int dir, const Arr4<P>& Cs, const Arr4<P>& Es, const typename P::T& A,
                        const typename P::T& Ad) {
  using T = typename P::T;
  QuarterPair<P> q;
  if (dir == 0) {  // ctmrg.jl:135-153
    const T &C1 = Cs[0], &C4 = Cs[3], &E1 = Es[0], &E3 = Es[2], &E4 = Es[3];
    T C1E1 = p.tc(C1, {-1, 1}, E1, {1, -2, -3, -4});
    T CEE4 = p.tc(C1E1, {1, -2, -5, -3}, E4, {1, -1, -6, -4});
    T CEEA = p.tc(CEE4, {-1, -2, -3, -4, 1, 2}, A, {1, 2, -5, -6, -7});
    T LU = p.tc(CEEA, {-1, -4, 1, 2, -2, -5, 3}, Ad, {1, 2, -3, -6, 3});
    q.R1 = p.rs(LU, {prod3(p, LU), -1});
    q.t1 = true;  // R1 = permutedims(reshape(LU, ...), (2, 1))
    T C4E3 = p.tc(C4, {-1, 1}, E3, {1, -2, -3, -4});
    T CEE4b = p.tc(C4E3, {1, -2, -6, -4}, E4, {-1, 1, -5, -3});
    T CEEAb = p.tc(CEE4b, {-1, -2, -3, -4, 1, 2}, A, {-5, 1, 2, -6, -7});
    T LB = p.tc(CEEAb, {-1, -4, 1, 2, -2, -5, 3}, Ad, {-3, 1, 2, -6, 3});
    q.R2 = p.rs(LB, {prod3(p, LB), -1});
  } else if (dir == 1) {  // ctmrg.jl:168-186
    const T &C2 = Cs[1], &C3 = Cs[2], &E1 = Es[0], &E2 = Es[1], &E3 = Es[2];
    T C2E1 = p.tc(C2, {1, -2}, E1, {-1, 1, -3, -4});
    T CEE2 = p.tc(C2E1, {-1, 1, -5, -3}, E2, {1, -2, -6, -4});
    T CEEA = p.tc(CEE2, {-1, -2, -3, -4, 1, 2}, A, {1, -5, -6, 2, -7});
    T RU = p.tc(CEEA, {-1, -4, 1, 2, -2, -5, 3}, Ad, {1, -3, -6, 2, 3});
    q.R1 = p.rs(RU, {prod3(p, RU), -1});
    T C3E3 = p.tc(C3, {-1, 1}, E3, {-2, 1, -3, -4});
    T CEE2b = p.tc(C3E3, {1, -2, -5, -3}, E2, {-1, 1, -6, -4});
    T CEEAb = p.tc(CEE2b, {-1, -2, -5, -6, 1, 2}, A, {-3, -4, 1, 2, -7});
    T RB = p.tc(CEEAb, {-1, -4, -2, -5, 1, 2, 3}, Ad, {-3, -6, 1, 2, 3});
    q.R2 = p.rs(RB, {prod3(p, RB), -1});
  } else if (dir == 2) {  // ctmrg.jl:201-219
    const T &C1 = Cs[0], &C2 = Cs[1], &E1 = Es[0], &E2 = Es[1], &E4 = Es[3];
    T C1E4 = p.tc(C1, {1, -2}, E4, {1, -1, -3, -4});
    T CEE1 = p.tc(C1E4, {-1, 1, -6, -4}, E1, {1, -2, -5, -3});
    T CEEA = p.tc(CEE1, {-1, -2, -5, -6, 1, 2}, A, {1, 2, -3, -4, -7});
    T UL = p.tc(CEEA, {-1, -4, -2, -5, 1, 2, 3}, Ad, {1, 2, -3, -6, 3});
    q.R1 = p.rs(UL, {prod3(p, UL), -1});
    T C2E2 = p.tc(C2, {-1, 1}, E2, {1, -2, -3, -4});
    T CEE1b = p.tc(C2E2, {1, -2, -6, -4}, E1, {-1, 1, -5, -3});
    T CEEAb = p.tc(CEE1b, {-1, -2, -5, -6, 1, 2}, A, {1, -3, -4, 2, -7});
    T UR = p.tc(CEEAb, {-1, -4, -2, -5, 1, 2, 3}, Ad, {1, -3, -6, 2, 3});
    q.R2 = p.rs(UR, {prod3(p, UR), -1});
  } else {  // ctmrg.jl:234-252
    const T &C3 = Cs[2], &C4 = Cs[3], &E2 = Es[1], &E3 = Es[2], &E4 = Es[3];
    T C4E4 = p.tc(C4, {1, -2}, E4, {-1, 1, -3, -4});
    T CEE3 = p.tc(C4E4, {-1, 1, -5, -3}, E3, {1, -2, -6, -4});
    T CEEA = p.tc(CEE3, {-1, -2, -5, -6, 1, 2}, A, {-3, 1, 2, -4, -7});
    T BL = p.tc(CEEA, {-1, -4, -2, -5, 1, 2, 3}, Ad, {-3, 1, 2, -6, 3});
    q.R1 = p.rs(BL, {prod3(p, BL), -1});
    T C3E2 = p.tc(C3, {1, -2}, E2, {-1, 1, -3, -4});
    T CEE3b = p.tc(C3E2, {-1, 1, -6, -4}, E3, {-2, 1, -5, -3});
    T CEEAb = p.tc(CEE3b, {-1, -2, -5, -6, 1, 2}, A, {-3, -4, 1, 2, -7});
    T BR = p.tc(CEEAb, {-1, -4, -2, -5, 1, 2, 3}, Ad, {-3, -6, 1, 2, 3});
    q.R2 = p.rs(BR, {prod3(p, BR), -1});
    q.t2 = true;  // R2 = permutedims(reshape(BR, ...), (2, 1))
  }
  return q;
}

// New edge tensor of a move.  The reference (ctmrg.jl:284-290 and the right,
// top and bottom analogues) forms T*A*A' (chi^2 D^6 elements) and then
// contracts Pd and P (2 chi^3 D^6 flops).  The same tensor
//   newE[c,c2,o,o'] = sum Pd[c,(a,g,g')] E[a,b,k,k'] A[..g..k..h..o..s] A'[..g'..k'..h'..o'..s] P[(b,h,h'),c2]
// is contracted here as ((Pd*E)*A)*A' then *P: 4 chi^3 D^4 + 4 chi^2 D^6 d
// flops, and chi^2 D^6 is never materialised.  Legs of A are (up, left,
// down, right, phys) = 0..4; lg/le/lh/lo are the legs grouped with Pd,
// contracted with E, grouped with P, and left open.
template <class P>
typename P::T proj_edge(P& p, const typename P::T& E, const typename P::T& A, const typename P::T& Ad,
                        const typename P::T& Pm, const typename P::T& Pd, int lg, int le, int lh, int lo) {
  using T = typename P::T;
  const int64_t chiE = p.dim(E, 0), chiB = p.dim(E, 1), D = p.dim(A, 0);
  T Pdr = p.rs(Pd, {p.dim(Pd, 0), chiE, D, D});
  T X2 = p.tc(Pdr, {-1, 1, -2, -3}, E, {1, -4, -5, -6});  // (c, g, g', b, k, k')
  std::vector<int> la(5), lad(5);
  la[lg] = 1;
  la[le] = 2;
  la[lh] = -5;
  la[lo] = -6;
  la[4] = -7;
  T X3 = p.tc(X2, {-1, 1, -2, -3, 2, -4}, A, la);  // (c, g', b, k', h, o, s)
  lad[lg] = 1;
  lad[le] = 2;
  lad[lh] = -5;
  lad[lo] = -6;
  lad[4] = 3;
  T X4 = p.tc(X3, {-1, 1, -2, 2, -3, -4, 3}, Ad, lad);  // (c, b, h, o, h', o')
  T Pr = p.rs(Pm, {chiB, D, D, p.dim(Pm, 1)});
  return p.tc(X4, {-1, 1, 2, -3, 3, -4}, Pr, {1, 2, 3, -2});  // (c, c2, o, o')
}

template <class P>
struct Projected {
  typename P::T Ca, E, Cb;  // unnormalised new tensors (order of up_*: left C1,E4,C4; right C2,E2,C3; top C1,E1,C2; bottom C4,E3,C3)
};

// proj_{left,right,top,bottom} (ctmrg.jl:267-375) with the cheaper edge order.
template <class P>
Projected<P> project(P& p, int dir, const Arr4<P>& Cs, const Arr4<P>& Es, const typename P::T& A,
                     const typename P::T& Ad, const typename P::T& Pm, const typename P::T& Pd) {
  using T = typename P::T;
  Projected<P> r;
  if (dir == 0) {  // ctmrg.jl:267-293
    T C1E1 = p.tc(Cs[0], {-2, 1}, Es[0], {1, -1, -3, -4});
    r.Ca = p.pm(p.mm(p.rs(C1E1, {p.dim(C1E1, 0), -1}), Pm), {1, 0});
    T C4E3 = p.tc(Cs[3], {-1, 1}, Es[2], {1, -4, -2, -3});
    r.Cb = p.mm(Pd, p.rs(C4E3, {-1, p.dim(C4E3, 3)}));
    r.E = proj_edge(p, Es[3], A, Ad, Pm, Pd, 0, 1, 2, 3);
  } else if (dir == 1) {  // ctmrg.jl:295-320
    T C2E1 = p.tc(Cs[1], {1, -2}, Es[0], {-1, 1, -3, -4});
    r.Ca = p.mm(p.rs(C2E1, {p.dim(C2E1, 0), -1}), Pm);
    T C3E3 = p.tc(Cs[2], {-1, 1}, Es[2], {-4, 1, -2, -3});
    r.Cb = p.mm(Pd, p.rs(C3E3, {-1, p.dim(C3E3, 3)}));
    r.E = proj_edge(p, Es[1], A, Ad, Pm, Pd, 0, 3, 2, 1);
  } else if (dir == 2) {  // ctmrg.jl:322-347
    T C1E4 = p.tc(Cs[0], {1, -2}, Es[3], {1, -1, -3, -4});
    r.Ca = p.mm(p.rs(C1E4, {p.dim(C1E4, 0), -1}), Pm);
    T C2E2 = p.tc(Cs[1], {-1, 1}, Es[1], {1, -4, -2, -3});
    r.Cb = p.mm(Pd, p.rs(C2E2, {-1, p.dim(C2E2, 3)}));
    r.E = proj_edge(p, Es[0], A, Ad, Pm, Pd, 1, 0, 3, 2);
  } else {  // ctmrg.jl:349-375
    T C4E4 = p.tc(Cs[3], {1, -2}, Es[3], {-1, 1, -3, -4});
    r.Ca = p.mm(p.rs(C4E4, {p.dim(C4E4, 0), -1}), Pm);
    T C3E2 = p.tc(Cs[2], {1, -1}, Es[1], {-4, 1, -2, -3});
    r.Cb = p.pm(p.mm(Pd, p.rs(C3E2, {-1, p.dim(C3E2, 3)})), {1, 0});
    r.E = proj_edge(p, Es[2], A, Ad, Pm, Pd, 1, 2, 3, 0);
  }
  return r;
}

// slots written by up_* (ctmrg.jl:377-491): corner a, corner b, edge
inline void move_slots(int dir, int* ia, int* ib, int* ie) {
  switch (dir) {
    case 0: *ia = 0; *ib = 3; *ie = 3; break;  // C1, C4, E4
    case 1: *ia = 1; *ib = 2; *ie = 1; break;  // C2, C3, E2
    case 2: *ia = 0; *ib = 1; *ie = 0; break;  // C1, C2, E1
    default: *ia = 3; *ib = 2; *ie = 2; break; // C4, C3, E3
  }
}

// evaluation.jl:169-200
template <class P>
typename P::T get_dm_h(P& p, const typename P::T& C1, const typename P::T& C2, const typename P::T& C3,
                       const typename P::T& C4, const typename P::T& E1l, const typename P::T& E1r,
                       const typename P::T& E2, const typename P::T& E3l, const typename P::T& E3r,
                       const typename P::T& E4, const typename P::T& Al, const typename P::T& Ar,
                       const typename P::T& Adl, const typename P::T& Adr) {
  using T = typename P::T;
  T C1E1 = p.tc(C1, {-1, 1}, E1l, {1, -2, -3, -4});
  T LU = p.tc(C1E1, {-1, -2, -3, 1}, Adl, {1, -4, -5, -6, -7});
  T C4E3 = p.tc(C4, {-1, 1}, E3l, {1, -2, -3, -4});
  T CEE4 = p.tc(E4, {-1, 1, -3, -5}, C4E3, {1, -2, -4, -6});
  T LB = p.tc(CEE4, {-1, -2, 1, 2, -4, -5}, Al, {-3, 1, 2, -6, -7});
  T L = p.tc(LB, {1, -2, 2, 3, 4, -3, -5}, LU, {1, -1, 2, 3, 4, -4, -6});
  T C2E1 = p.tc(C2, {1, -2}, E1r, {-1, 1, -3, -4});
  T RU = p.tc(C2E1, {-1, -2, 1, -3}, Ar, {1, -4, -5, -6, -7});
  T C3E3 = p.tc(C3, {-1, 1}, E3r, {-2, 1, -3, -4});
  T CEE2 = p.tc(C3E3, {1, -2, -3, -5}, E2, {-1, 1, -4, -6});
  T RB = p.tc(CEE2, {-1, -2, -3, -4, 1, 2}, Adr, {-5, -6, 1, 2, -7});
  T R = p.tc(RU, {-1, 1, 2, -3, 3, 4, -5}, RB, {1, -2, 3, 4, 2, -4, -6});
  T roh = p.tc(L, {1, 2, 3, 4, -1, -3}, R, {1, 2, 3, 4, -2, -4});
  const int64_t d = p.dim(Al, 4);
  return p.rs(roh, {d * d, d * d});
}

// evaluation.jl:217-248
template <class P>
typename P::T get_dm_v(P& p, const typename P::T& C1, const typename P::T& C2, const typename P::T& C3,
                       const typename P::T& C4, const typename P::T& E1, const typename P::T& E2u,
                       const typename P::T& E2d, const typename P::T& E3, const typename P::T& E4u,
                       const typename P::T& E4d, const typename P::T& Au, const typename P::T& Ad,
                       const typename P::T& Adu, const typename P::T& Add) {
  using T = typename P::T;
  T C1E1 = p.tc(C1, {-1, 1}, E1, {1, -2, -3, -4});
  T CEE4 = p.tc(C1E1, {1, -2, -3, -5}, E4u, {1, -1, -4, -6});
  T UL = p.tc(CEE4, {-1, -2, 1, 2, -3, -4}, Au, {1, 2, -5, -6, -7});
  T C2E2 = p.tc(C2, {-1, 1}, E2u, {1, -2, -3, -4});
  T UR = p.tc(C2E2, {-1, -2, -3, 1}, Adu, {-4, -5, -6, 1, -7});
  T U = p.tc(UL, {-1, 1, 3, 4, -3, 2, -5}, UR, {1, -2, 2, 3, 4, -4, -6});
  T C4E3 = p.tc(C4, {-1, 1}, E3, {1, -2, -3, -4});
  T CEE4b = p.tc(C4E3, {1, -2, -4, -6}, E4d, {-1, 1, -3, -5});
  T BL = p.tc(CEE4b, {-1, -2, -3, -4, 1, 2}, Add, {-5, 1, 2, -6, -7});
  T C3E2 = p.tc(C3, {1, -2}, E2d, {-1, 1, -3, -4});
  T BR = p.tc(C3E2, {-1, -2, 1, -3}, Ad, {-4, -5, -6, 1, -7});
  T B = p.tc(BL, {-1, 1, 2, 3, -4, 4, -6}, BR, {-2, 1, 4, -3, 2, 3, -5});
  T rov = p.tc(U, {1, 2, 3, 4, -1, -3}, B, {1, 2, 3, 4, -2, -4});
  const int64_t d = p.dim(Au, 4);
  return p.rs(rov, {d * d, d * d});
}

// evaluation.jl:501-518: each Ad with its factor of the plaquette MPO
// [s1, s2, s3, s4] (get_local_h), virtual and Hamiltonian bonds fused
template <class P>
Arr4<P> get_op_Ad4(P& p, const Arr4<P>& s, const Arr4<P>& Ad) {
  using T = typename P::T;
  Arr4<P> op;
  T o1 = p.tc(s[0], {-6, 1, -4}, Ad[0], {-1, -2, -3, -5, 1});
  op[0] = p.rs(o1, {p.dim(o1, 0), p.dim(o1, 1), p.dim(o1, 2), p.dim(o1, 3) * p.dim(o1, 4), p.dim(o1, 5)});
  T o2 = p.tc(s[1], {-2, -7, 1, -4}, Ad[1], {-1, -3, -5, -6, 1});
  op[1] = p.rs(o2, {p.dim(o2, 0), p.dim(o2, 1) * p.dim(o2, 2), p.dim(o2, 3) * p.dim(o2, 4), p.dim(o2, 5),
                    p.dim(o2, 6)});
  T o3 = p.tc(s[2], {-1, -7, 1, -3}, Ad[2], {-2, -4, -5, -6, 1});
  op[2] = p.rs(o3, {p.dim(o3, 0) * p.dim(o3, 1), p.dim(o3, 2) * p.dim(o3, 3), p.dim(o3, 4), p.dim(o3, 5),
                    p.dim(o3, 6)});
  T o4 = p.tc(s[3], {-4, -6, 1}, Ad[3], {-1, -2, -3, -5, 1});
  op[3] = p.rs(o4, {p.dim(o4, 0), p.dim(o4, 1), p.dim(o4, 2), p.dim(o4, 3) * p.dim(o4, 4), p.dim(o4, 5)});
  return op;
}

template <class P>
typename P::T fuse3(P& p, const typename P::T& x) {
  return p.rs(x, {prod3(p, x), -1});
}

// evaluation.jl:443-498: energy and norm of the 2 x 2 cluster (plaquette)
//   C1 - E1l - E1r - C2
//   E4u - A1 -- A2 - E2u
//   E4d - A4 -- A3 - E2d
//   C4 - E3l - E3r - C3
template <class P>
std::array<typename P::T, 2> energy_norm_4x4(P& p, const typename P::T& C1, const typename P::T& C2,
                                              const typename P::T& C3, const typename P::T& C4,
                                              const typename P::T& E1l, const typename P::T& E1r,
                                              const typename P::T& E2u, const typename P::T& E2d,
                                              const typename P::T& E3l, const typename P::T& E3r,
                                              const typename P::T& E4u, const typename P::T& E4d, const Arr4<P>& A,
                                              const Arr4<P>& Ad, const Arr4<P>& op) {
  using T = typename P::T;
  T C1E1 = p.tc(C1, {-1, 1}, E1l, {1, -2, -3, -4});
  T CEE4 = p.tc(C1E1, {1, -2, -5, -3}, E4u, {1, -1, -6, -4});
  T CEEA1 = p.tc(CEE4, {-1, -2, -3, -4, 1, 2}, A[0], {1, 2, -5, -6, -7});
  T eLU = fuse3(p, p.tc(CEEA1, {-1, -4, 1, 2, -2, -5, 3}, op[0], {1, 2, -3, -6, 3}));
  T nLU = fuse3(p, p.tc(CEEA1, {-1, -4, 1, 2, -2, -5, 3}, Ad[0], {1, 2, -3, -6, 3}));

  T C4E3 = p.tc(C4, {-1, 1}, E3l, {1, -2, -3, -4});
  T CEE4b = p.tc(C4E3, {1, -2, -6, -4}, E4d, {-1, 1, -5, -3});
  T CEEA4 = p.tc(CEE4b, {-1, -2, -3, -4, 1, 2}, A[3], {-5, 1, 2, -6, -7});
  T eLB = fuse3(p, p.tc(CEEA4, {-1, -4, 1, 2, -2, -5, 3}, op[3], {-3, 1, 2, -6, 3}));
  T nLB = fuse3(p, p.tc(CEEA4, {-1, -4, 1, 2, -2, -5, 3}, Ad[3], {-3, 1, 2, -6, 3}));

  T C2E1 = p.tc(C2, {1, -2}, E1r, {-1, 1, -3, -4});
  T CEE2 = p.tc(C2E1, {-1, 1, -5, -3}, E2u, {1, -2, -6, -4});
  T CEEA2 = p.tc(CEE2, {-1, -2, -3, -4, 1, 2}, A[1], {1, -5, -6, 2, -7});
  T eRU = fuse3(p, p.tc(CEEA2, {-1, -4, 1, 2, -2, -5, 3}, op[1], {1, -3, -6, 2, 3}));
  T nRU = fuse3(p, p.tc(CEEA2, {-1, -4, 1, 2, -2, -5, 3}, Ad[1], {1, -3, -6, 2, 3}));

  T C3E3 = p.tc(C3, {-1, 1}, E3r, {-2, 1, -3, -4});
  T CEE2b = p.tc(C3E3, {1, -2, -5, -3}, E2d, {-1, 1, -6, -4});
  T CEEA3 = p.tc(CEE2b, {-1, -2, -5, -6, 1, 2}, A[2], {-3, -4, 1, 2, -7});
  T eRB = fuse3(p, p.tc(CEEA3, {-1, -4, -2, -5, 1, 2, 3}, op[2], {-3, -6, 1, 2, 3}));
  T nRB = fuse3(p, p.tc(CEEA3, {-1, -4, -2, -5, 1, 2, 3}, Ad[2], {-3, -6, 1, 2, 3}));

  T eL = p.tc(p.pm(eLU, {1, 0}), {-1, 1}, eLB, {1, -2});
  T eR = p.tc(eRU, {-1, 1}, eRB, {1, -2});
  T nL = p.tc(p.pm(nLU, {1, 0}), {-1, 1}, nLB, {1, -2});
  T nR = p.tc(nRU, {-1, 1}, nRB, {1, -2});
  return {p.tc(eL, {1, 2}, eR, {1, 2}), p.tc(nL, {1, 2}, nR, {1, 2})};
}

// The arguments of energy_norm_4x4 for get_es_energy_4x4 (evaluation.jl:358-398):
// the nested environment with the phase shifts of the sites right of (px) and
// below (py) the first
template <class P, class Shift>
std::array<typename P::T, 2> es_plaquette(P& p, Shift sh, const Arr4<P>& s, const typename P::T& A,
                                          const typename P::T& Ad, Arr4<P> C, const Arr4<P>& E, double px,
                                          double py) {
  using T = typename P::T;
  T E1r = sh(E[0], px);
  T A2 = sh(A, px), A2d = sh(Ad, px);
  T A3 = sh(A, px), A3d = sh(Ad, px);
  T E3r = sh(E[2], px);
  C[1] = sh(C[1], px);
  C[2] = sh(C[2], px);
  T E2u = sh(E[1], px), E2d = sh(E[1], px);
  C[3] = sh(C[3], py);
  C[2] = sh(C[2], py);
  T E3l = sh(E[2], py);
  E3r = sh(E3r, py);
  T E4d = sh(E[3], py);
  E2d = sh(E2d, py);
  T A4 = sh(A, py), A4d = sh(Ad, py);
  A3 = sh(A3, py);
  A3d = sh(A3d, py);
  Arr4<P> As{A, A2, A3, A4}, Ads{Ad, A2d, A3d, A4d};
  Arr4<P> op = get_op_Ad4(p, s, Ads);
  return energy_norm_4x4(p, C[0], C[1], C[2], C[3], E[0], E1r, E2u, E2d, E3l, E3r, E[3], E4d, As, Ads, op);
}

// evaluation.jl:110-122
template <class P>
typename P::T get_single_dm(P& p, const typename P::T& C1, const typename P::T& C2, const typename P::T& C3,
                            const typename P::T& C4, const typename P::T& E1, const typename P::T& E2,
                            const typename P::T& E3, const typename P::T& E4) {
  using T = typename P::T;
  T C1E1 = p.tc(C1, {-1, 1}, E1, {1, -2, -3, -4});
  T CEC2 = p.tc(C1E1, {-1, 1, -3, -4}, C2, {1, -2});
  T CECE4 = p.tc(CEC2, {1, -2, -3, -5}, E4, {1, -1, -4, -6});
  T C4E3 = p.tc(C4, {-1, 1}, E3, {1, -2, -3, -4});
  T CEC3 = p.tc(C4E3, {-1, 1, -3, -4}, C3, {-2, 1});
  T CECE2 = p.tc(CEC3, {-1, 1, -3, -5}, E2, {-2, 1, -4, -6});
  return p.tc(CECE4, {1, 2, -1, -2, -5, -6}, CECE2, {1, 2, -3, -4, -7, -8});
}

}  // namespace ipeps
