// oracle.cpp -- CPU restatement of shtensor's single-rank block-sparse contraction.
//
// TEST INFRASTRUCTURE ONLY (the checker).  Loaded by tests/, __graft_entry__.smoke() and
// bench.py's CPU legs; the product library never links or calls it.  Built with
// -ffp-contract=off so that every fused multiply-add below is an explicit std::fma.
//
// Reference citations are relative to the shtensor project root.
#include "oracle.h"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <numeric>
#include <set>
#include <stdexcept>
#include <string>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

#include "oracle_internal.h"

namespace ora {

static void set_err(char* err, int errlen, const std::string& msg) {
  if (err && errlen > 0) {
    std::snprintf(err, (size_t)errlen, "%s", msg.c_str());
  }
}

// ---------------------------------------------------------------------------------------
// Einsum -> matrix maps.  Restates compute_contract_info, ContractInfo.h:69-346:
//  * tokens: index runs of [A-Za-z_], ',' and '->', whitespace skipped (:100-146);
//  * syntax INDICES , INDICES -> INDICES (:160-215);
//  * axis ids by first appearance over A, then B, then C (:175-184);
//  * con = A∩B, ncon1 = A\con, ncon2 = B\con, each ordered by axis id (:233-243);
//  * A rows = ncon1, A cols = con, B rows = con, B cols = ncon2, C rows = ncon1,
//    C cols = ncon2, as local positions (:266-291);
//  * size checks A-rows vs C-rows, B-cols vs C-cols, A-cols vs B-rows (:293-328).
// Two checks are added where the reference silently mis-maps: the number of indices of a
// tensor must equal its order, and C's indices must be exactly ncon1 ∪ ncon2 (the
// reference's std::map lookup returns position 0 for a missing index, :266-279).
// ---------------------------------------------------------------------------------------
bool parse_contraction(const std::string& expr, int nA, const int* sA, int nB, const int* sB,
                       int nC, const int* sC, Maps& m, std::string& err) {
  if (expr.empty()) { err = "Equation is empty"; return false; }
  struct Tok { int type; int pos; std::string val; };  // 0 idx, 1 comma, 2 arrow
  std::vector<Tok> toks;
  auto valid = [](char c) { return std::isalpha((unsigned char)c) || c == '_'; };
  const int L = (int)expr.size();
  for (int pos = 0; pos < L; ++pos) {
    const char c = expr[pos];
    if (std::isspace((unsigned char)c)) continue;
    if (valid(c)) {
      std::string s;
      int p = pos;
      while (p < L && valid(expr[p])) s += expr[p++];
      toks.push_back({0, pos, s});
      pos = p - 1;
      continue;
    }
    if (c == '-' && pos + 1 < L && expr[pos + 1] == '>') { toks.push_back({2, pos, "->"}); ++pos; continue; }
    if (c == ',') { toks.push_back({1, pos, ","}); continue; }
    char buf[96];
    std::snprintf(buf, sizeof buf, "Unknown character in equation at position %d: %c", pos, c);
    err = buf;
    return false;
  }
  const int want[5] = {0, 1, 0, 2, 0};
  const char* names[3] = {"index", ",", "->"};
  for (int i = 0; i < 5; ++i) {
    if (i >= (int)toks.size()) { err = std::string("Unexpected end of expression, expected ") + names[want[i]]; return false; }
    if (toks[i].type != want[i]) {
      char buf[96];
      std::snprintf(buf, sizeof buf, "Expected %s at position %d", names[want[i]], toks[i].pos);
      err = buf;
      return false;
    }
  }
  if (toks.size() != 5) { err = "Invalid syntax"; return false; }

  std::map<char, int> axis;
  int next = 0;
  auto to_axes = [&](const std::string& s) {
    std::vector<int> out;
    for (char c : s) {
      if (!axis.count(c)) axis[c] = next++;
      out.push_back(axis[c]);
    }
    return out;
  };
  const std::vector<int> ia = to_axes(toks[0].val), ib = to_axes(toks[2].val), ic = to_axes(toks[4].val);
  const std::set<int> sa(ia.begin(), ia.end()), sb(ib.begin(), ib.end()), sc(ic.begin(), ic.end());
  if (sa.size() != ia.size() || sb.size() != ib.size() || sc.size() != ic.size()) {
    err = "Duplicate tensor indices"; return false;
  }
  std::set<int> con, n1, n2;
  std::set_intersection(sa.begin(), sa.end(), sb.begin(), sb.end(), std::inserter(con, con.begin()));
  std::set_difference(sa.begin(), sa.end(), con.begin(), con.end(), std::inserter(n1, n1.begin()));
  std::set_difference(sb.begin(), sb.end(), con.begin(), con.end(), std::inserter(n2, n2.begin()));
  if (n1.empty() || n2.empty()) { err = "Element-wise multiplication not supported"; return false; }
  if (con.empty()) { err = "No indices found over which to contract"; return false; }
  if (n1.size() + n2.size() != sc.size()) { err = "Dimension mismatch"; return false; }
  std::set<int> freeset(n1);
  freeset.insert(n2.begin(), n2.end());
  if (freeset != sc) { err = "Output indices must be the free indices of both inputs"; return false; }
  if ((int)ia.size() != nA || (int)ib.size() != nB || (int)ic.size() != nC) {
    err = "Number of indices does not match tensor order"; return false;
  }
  auto local = [](const std::vector<int>& all, const std::set<int>& sel) {
    std::vector<int> out;
    for (int g : sel) out.push_back((int)(std::find(all.begin(), all.end(), g) - all.begin()));
    return out;
  };
  m.rowA = local(ia, n1); m.colA = local(ia, con);
  m.rowB = local(ib, con); m.colB = local(ib, n2);
  m.rowC = local(ic, n1); m.colC = local(ic, n2);
  auto check = [&](const std::vector<int>& m1, const std::vector<int>& m2, const int* d1,
                   const int* d2, const char* n1s, const char* n2s) {
    for (size_t i = 0; i < m1.size(); ++i) {
      if (d1 && d2 && d1[m1[i]] != d2[m2[i]]) {
        char buf[160];
        std::snprintf(buf, sizeof buf,
                      "Sizes for dimensions %d in %s and for dimension %d in %s do not match.",
                      m1[i], n1s, m2[i], n2s);
        err = buf;
        return false;
      }
    }
    return true;
  };
  if (!check(m.rowA, m.rowC, sA, sC, "tensor A", "tensor C")) return false;
  if (!check(m.colB, m.colC, sB, sC, "tensor B", "tensor C")) return false;
  if (!check(m.colA, m.rowB, sA, sB, "tensor A", "tensor B")) return false;
  return true;
}

// Column-major strides, Utils.h:81-94.
std::vector<int64_t> strides_of(const int* sizes, int n) {
  std::vector<int64_t> s(n);
  int64_t acc = 1;
  for (int i = 0; i < n; ++i) { s[i] = acc; acc *= sizes[i]; }
  return s;
}

// create_scatter_vector, ContractInfo.h:38-66: element offset of each matrix index built
// from the listed axes, the first listed axis varying fastest.
std::vector<int64_t> scatter_of(const std::vector<int>& map, const int* sizes, int n) {
  int64_t total = 1;
  for (int ax : map) total *= sizes[ax];
  const std::vector<int64_t> st = strides_of(sizes, n);
  std::vector<int64_t> out((size_t)total, 0);
  for (int64_t idx = 0; idx < total; ++idx) {
    int64_t s = 1, v = 0;
    for (int ax : map) { v += ((idx / s) % sizes[ax]) * st[ax]; s *= sizes[ax]; }
    out[(size_t)idx] = v;
  }
  return out;
}

// Bytewise "is +0.0" test of the XMM kernel (KernelImpl.cpp:462-463 sums the bytes).
template <typename T>
static bool bytes_zero(T v) {
  unsigned char b[sizeof(T)];
  std::memcpy(b, &v, sizeof(T));
  for (unsigned char x : b) if (x) return false;
  return true;
}

// One (A,B,C) block triple in the XMM kernel's arithmetic order, KernelImpl.cpp:553-735:
// j (columns) -> i (rows) -> k ascending; c = beta*c (or 0 when beta is +0.0, :594-619);
// per k: a = alpha*a (vmulpd), c = fma(a, b, c) (vfmadd231pd, AvxHelper.cpp:287).
// The C address is scatter_row[i] + scatter_col[j] for every layout.  (The JIT uses the
// matrix index i + j*m for C whenever C's row map is 0..r-1, which equals the scatter
// address only when C's column map is ascending as well.)
template <typename T>
void xmm_triple(const T* a, const T* b, T* c, const std::vector<int64_t>& rA,
                const std::vector<int64_t>& cA, const std::vector<int64_t>& rB,
                const std::vector<int64_t>& cB, const std::vector<int64_t>& rC,
                const std::vector<int64_t>& cC, T alpha, T beta, bool apply_beta) {
  const int64_t m = (int64_t)rA.size(), n = (int64_t)cB.size(), k = (int64_t)cA.size();
  const bool bz = bytes_zero(beta), az = bytes_zero(alpha);
  for (int64_t j = 0; j < n; ++j) {
    for (int64_t i = 0; i < m; ++i) {
      T* pc = c + rC[i] + cC[j];
      T acc = *pc;
      if (apply_beta) acc = bz ? T(0) : beta * acc;
      if (!az) {
        for (int64_t l = 0; l < k; ++l) {
          const T av = alpha * a[rA[i] + cA[l]];
          acc = std::fma(av, b[rB[l] + cB[j]], acc);
        }
      }
      *pc = acc;
    }
  }
}
template void xmm_triple<double>(const double*, const double*, double*, const std::vector<int64_t>&,
                                 const std::vector<int64_t>&, const std::vector<int64_t>&,
                                 const std::vector<int64_t>&, const std::vector<int64_t>&,
                                 const std::vector<int64_t>&, double, double, bool);

// Utils::reshape, Utils.h:315-359: out[rolled(order-permuted index)] = in[i].
template <typename T>
void reshape(const T* in, const int* sizes, const int* order, int n, T* out);
template <>
void reshape<double>(const double* in, const int* sizes, const int* order, int n, double* out) {
  std::vector<int> rs(n);
  for (int i = 0; i < n; ++i) rs[i] = sizes[order[i]];
  const std::vector<int64_t> ss = strides_of(sizes, n), rst = strides_of(rs.data(), n);
  int64_t total = 1;
  for (int i = 0; i < n; ++i) total *= sizes[i];
  std::vector<int64_t> si(n);
  for (int64_t s = 0; s < total; ++s) {
    int64_t t = s;
    for (int i = n - 1; i >= 0; --i) { si[i] = t / ss[i]; t %= ss[i]; }
    int64_t r = 0;
    for (int i = 0; i < n; ++i) r += si[order[i]] * rst[i];
    out[r] = in[s];
  }
}

// Netlib reference DGEMM('N','N') loop order: j -> (beta on column) -> l -> i.
static void gemm_nn_ref(int m, int n, int k, double alpha, const double* A, int lda,
                        const double* B, int ldb, double beta, double* C, int ldc) {
  for (int j = 0; j < n; ++j) {
    if (beta == 0.0) {
      for (int i = 0; i < m; ++i) C[i + (int64_t)j * ldc] = 0.0;
    } else if (beta != 1.0) {
      for (int i = 0; i < m; ++i) C[i + (int64_t)j * ldc] = beta * C[i + (int64_t)j * ldc];
    }
    for (int l = 0; l < k; ++l) {
      const double t = alpha * B[l + (int64_t)j * ldb];
      for (int i = 0; i < m; ++i) C[i + (int64_t)j * ldc] = C[i + (int64_t)j * ldc] + t * A[i + (int64_t)l * lda];
    }
  }
}

// The LAPACK path of KernelImpl.cpp:142-208 on one triple, with a pluggable GEMM.
void lapack_triple(const double* a, const double* b, double* c, const int* sA, int nA,
                   const int* sB, int nB, const int* sC, int nC, const Maps& m, double alpha,
                   double beta, GemmFn gemm, ReshapeFn rfn, std::vector<double>& buf) {
  if (!rfn) rfn = reshape<double>;
  std::vector<int> oa(m.rowA), ob(m.rowB), oc(m.rowC);
  oa.insert(oa.end(), m.colA.begin(), m.colA.end());
  ob.insert(ob.end(), m.colB.begin(), m.colB.end());
  oc.insert(oc.end(), m.colC.begin(), m.colC.end());
  int64_t za = 1, zb = 1, zc = 1;
  for (int i = 0; i < nA; ++i) za *= sA[i];
  for (int i = 0; i < nB; ++i) zb *= sB[i];
  for (int i = 0; i < nC; ++i) zc *= sC[i];
  buf.resize((size_t)(za + zb + zc));
  double* pa = buf.data();
  double* pb = pa + za;
  double* pc = pb + zb;
  rfn(a, sA, oa.data(), nA, pa);
  rfn(b, sB, ob.data(), nB, pb);
  rfn(c, sC, oc.data(), nC, pc);
  int mm = 1, nn = 1, kk = 1;
  for (int ax : m.rowA) mm *= sA[ax];
  for (int ax : m.colB) nn *= sB[ax];
  for (int ax : m.colA) kk *= sA[ax];
  (gemm ? gemm : gemm_nn_ref)(mm, nn, kk, alpha, pa, mm, pb, kk, beta, pc, mm);
  std::vector<int> ocr(nC), scr(nC);
  for (int i = 0; i < nC; ++i) { ocr[oc[i]] = i; scr[i] = sC[oc[i]]; }
  rfn(pc, scr.data(), ocr.data(), nC, c);
}

// ---------------------------------------------------------------------------------------
// Block norms, BlockSpan.h:140-164.
// FROBENIUS and MAXABS use the canonical deterministic order shared with the device
// kernels: chunks of 4096 consecutive elements; in chunk c, 128 lane values
// p[j] = op(p[j], v_e) over e = c*4096 + j + 128*i ascending (FROBENIUS: fma(v, v, p),
// MAXABS: max(p, |v|)); then p[j] op= p[j+h] for h = 64, 32, ..., 1; the chunk values are
// folded in ascending order starting from chunk 0; FROBENIUS ends with sqrt.
// FROBENIUS_REFCOMPAT reproduces the reference's int accumulator: acc = int(acc + v*v).
// ---------------------------------------------------------------------------------------
double block_norm(const double* d, int64_t n, int norm) {
  if (norm == 2) {
    int acc = 0;
    for (int64_t i = 0; i < n; ++i) acc = (int)((double)acc + d[i] * d[i]);
    return std::sqrt((double)acc);
  }
  const bool maxabs = norm == 1;
  const int64_t chunk = 4096;
  const int lanes = 128;
  double total = 0.0;
  for (int64_t c = 0; c * chunk < n; ++c) {
    double p[lanes];
    for (int j = 0; j < lanes; ++j) p[j] = 0.0;
    const int64_t base = c * chunk, end = std::min(n, base + chunk);
    for (int64_t e = base; e < end; ++e) {
      const int j = (int)((e - base) % lanes);
      p[j] = maxabs ? std::max(p[j], std::fabs(d[e])) : std::fma(d[e], d[e], p[j]);
    }
    for (int h = lanes / 2; h >= 1; h >>= 1)
      for (int j = 0; j < h; ++j) p[j] = maxabs ? std::max(p[j], p[j + h]) : p[j] + p[j + h];
    total = c == 0 ? p[0] : (maxabs ? std::max(total, p[0]) : total + p[0]);
  }
  return maxabs ? total : std::sqrt(total);
}

// ---------------------------------------------------------------------------------------
// Storage layout, BaseTensor.cpp:117-251 (single rank, every block local):
//  id = Σ_d idx_d · gridstride_d with column-major grid strides (:172-178);
//  blocks sorted by id (:181-195); offsets = running element count in that order
//  (:213-232); rows[r] = Σ_{r'<r} (#blocks whose mode-0 index is r') (:200-208).
//  The sort is over all ids, so rows[] is a count prefix and does not delimit the blocks of
//  mode-0 index r whenever another mode has more than one block; it is kept for parity.
// ---------------------------------------------------------------------------------------
bool reserve(int order, const int* nblk, const int* bsizes, int64_t n, const int* idx,
             BTensor& t, std::string& err) {
  t.order = order;
  t.nblk.assign(nblk, nblk + order);
  t.bs.assign(order, {});
  int pos = 0;
  for (int d = 0; d < order; ++d) { t.bs[d].assign(bsizes + pos, bsizes + pos + nblk[d]); pos += nblk[d]; }
  t.gstride = strides_of(nblk, order);
  std::vector<int64_t> rolled((size_t)n, 0);
  std::vector<int64_t> rowcount((size_t)nblk[0], 0);
  for (int64_t b = 0; b < n; ++b) {
    for (int d = 0; d < order; ++d) {
      const int v = idx[(int64_t)d * n + b];
      if (v < 0 || v >= nblk[d]) { err = "reserve: block index out of range"; return false; }
      rolled[(size_t)b] += (int64_t)v * t.gstride[d];
    }
    rowcount[(size_t)idx[b]]++;
  }
  std::sort(rolled.begin(), rolled.end());
  if (std::adjacent_find(rolled.begin(), rolled.end()) != rolled.end()) {
    err = "reserve: duplicate block index"; return false;
  }
  t.ids = rolled;
  t.rows.assign((size_t)nblk[0], 0);
  int64_t acc = 0;
  for (int r = 0; r < nblk[0]; ++r) { t.rows[(size_t)r] = acc; acc += rowcount[(size_t)r]; }
  t.offsets.resize((size_t)n);
  int64_t off = 0;
  for (int64_t b = 0; b < n; ++b) { t.offsets[(size_t)b] = off; off += t.block_size(t.ids[(size_t)b]); }
  t.nnz = off;
  return true;
}

int64_t BTensor::block_size(int64_t id) const {
  int64_t s = 1;
  for (int d = 0; d < order; ++d) { s *= bs[d][(size_t)((id / gstride[d]) % nblk[d])]; }
  return s;
}
void BTensor::block_dims(int64_t id, int* dims) const {
  for (int d = 0; d < order; ++d) dims[d] = bs[d][(size_t)((id / gstride[d]) % nblk[d])];
}
void BTensor::block_coords(int64_t id, int* c) const {
  for (int d = 0; d < order; ++d) c[d] = (int)((id / gstride[d]) % nblk[d]);
}

void load_tensor(int order, const int* nblk, const int* bsizes, int64_t n, const int64_t* ids,
                 const int64_t* offs, BTensor& t) {
  t.order = order;
  t.nblk.assign(nblk, nblk + order);
  t.bs.assign(order, {});
  int pos = 0;
  for (int d = 0; d < order; ++d) { t.bs[d].assign(bsizes + pos, bsizes + pos + nblk[d]); pos += nblk[d]; }
  t.gstride = strides_of(nblk, order);
  t.ids.assign(ids, ids + n);
  t.offsets.assign(offs, offs + n);
  t.nnz = 0;
  for (int64_t b = 0; b < n; ++b) t.nnz = std::max(t.nnz, offs[b] + t.block_size(ids[b]));
}

// ---------------------------------------------------------------------------------------
// Block-sparse contraction (absent from the reference; canonical rules of this project):
//  1. pairs: stored A block a and B block b whose contracted-mode block indices agree;
//     the C block takes A's free block indices and B's free block indices at C's modes;
//  2. screening: keep the pair iff eps <= 0 or norm(a)*norm(b) >= eps;
//  3. pair order: ascending (idC, idA, idB);
//  4. result pattern: sorted union of C's stored ids and the pairs' idC; new blocks start
//     zero-filled (reserve zero-fills, BaseTensor.cpp:238-239);
//  5. values: every result block gets c = beta*c once (0 when beta is +0.0), then each pair
//     in order adds alpha*A*B in the XMM order (k ascending, fma); alpha == +0.0 skips.
// ---------------------------------------------------------------------------------------
bool contract(const std::string& expr, double alpha, const BTensor& A, const double* dA,
              const BTensor& B, const double* dB, double beta, const BTensor& Cin,
              const double* dCin, double eps, int norm, int lapack_blocks, int nthreads,
              GemmFn gemm, ReshapeFn rfn, ContractResult& R, std::string& err) {
  std::vector<int> sA(A.order), sB(B.order), sC(Cin.order);
  Maps m;
  if (!parse_contraction(expr, A.order, nullptr, B.order, nullptr, Cin.order, nullptr, m, err)) return false;
  // block-size lists of matched modes must agree
  auto same = [](const std::vector<int>& x, const std::vector<int>& y) { return x == y; };
  for (size_t t = 0; t < m.rowA.size(); ++t)
    if (!same(A.bs[m.rowA[t]], Cin.bs[m.rowC[t]])) { err = "Block sizes of tensor A and tensor C do not match"; return false; }
  for (size_t t = 0; t < m.colB.size(); ++t)
    if (!same(B.bs[m.colB[t]], Cin.bs[m.colC[t]])) { err = "Block sizes of tensor B and tensor C do not match"; return false; }
  for (size_t t = 0; t < m.colA.size(); ++t)
    if (!same(A.bs[m.colA[t]], B.bs[m.rowB[t]])) { err = "Block sizes of tensor A and tensor B do not match"; return false; }

  const auto t0 = std::chrono::steady_clock::now();
  const int64_t nA = (int64_t)A.ids.size(), nB = (int64_t)B.ids.size();
  std::vector<double> normA, normB;
  if (eps > 0.0) {
    normA.resize((size_t)nA);
    normB.resize((size_t)nB);
    for (int64_t i = 0; i < nA; ++i) normA[(size_t)i] = block_norm(dA + A.offsets[(size_t)i], A.block_size(A.ids[(size_t)i]), norm);
    for (int64_t i = 0; i < nB; ++i) normB[(size_t)i] = block_norm(dB + B.offsets[(size_t)i], B.block_size(B.ids[(size_t)i]), norm);
  }
  // keys over the contracted modes, C-id parts over the free modes
  std::vector<int> cA(A.order), cB(B.order);
  auto keyof = [&](const std::vector<int>& coords, const std::vector<int>& modes, const BTensor& T) {
    int64_t k = 0, s = 1;
    for (int ax : modes) { k += coords[ax] * s; s *= T.nblk[ax]; }
    return k;
  };
  std::vector<int64_t> keyA((size_t)nA), partA((size_t)nA), keyB((size_t)nB), partB((size_t)nB);
  for (int64_t i = 0; i < nA; ++i) {
    A.block_coords(A.ids[(size_t)i], cA.data());
    keyA[(size_t)i] = keyof(cA, m.colA, A);
    int64_t p = 0;
    for (size_t t = 0; t < m.rowA.size(); ++t) p += (int64_t)cA[m.rowA[t]] * Cin.gstride[m.rowC[t]];
    partA[(size_t)i] = p;
  }
  std::multimap<int64_t, int64_t> bykey;
  for (int64_t i = 0; i < nB; ++i) {
    B.block_coords(B.ids[(size_t)i], cB.data());
    keyB[(size_t)i] = keyof(cB, m.rowB, B);
    int64_t p = 0;
    for (size_t t = 0; t < m.colB.size(); ++t) p += (int64_t)cB[m.colB[t]] * Cin.gstride[m.colC[t]];
    partB[(size_t)i] = p;
    bykey.emplace(keyB[(size_t)i], i);  // multimap keeps insertion order among equal keys
  }
  std::vector<Pair> pairs;
  for (int64_t a = 0; a < nA; ++a) {
    auto rng = bykey.equal_range(keyA[(size_t)a]);
    for (auto it = rng.first; it != rng.second; ++it) {
      const int64_t b = it->second;
      if (eps > 0.0 && !(normA[(size_t)a] * normB[(size_t)b] >= eps)) continue;
      pairs.push_back({partA[(size_t)a] + partB[(size_t)b], a, b});
    }
  }
  std::sort(pairs.begin(), pairs.end(), [](const Pair& x, const Pair& y) {
    if (x.c != y.c) return x.c < y.c;
    if (x.a != y.a) return x.a < y.a;
    return x.b < y.b;
  });
  // result pattern
  std::vector<int64_t> ids(Cin.ids);
  for (const Pair& p : pairs) ids.push_back(p.c);
  std::sort(ids.begin(), ids.end());
  ids.erase(std::unique(ids.begin(), ids.end()), ids.end());
  BTensor& C = R.C;
  C.order = Cin.order; C.nblk = Cin.nblk; C.bs = Cin.bs; C.gstride = Cin.gstride;
  C.ids = ids;
  C.offsets.resize(ids.size());
  int64_t off = 0;
  for (size_t i = 0; i < ids.size(); ++i) { C.offsets[i] = off; off += C.block_size(ids[i]); }
  C.nnz = off;
  C.rows.assign((size_t)C.nblk[0], 0);
  {
    std::vector<int64_t> cnt((size_t)C.nblk[0], 0);
    for (int64_t id : ids) cnt[(size_t)(id % C.nblk[0])]++;
    int64_t acc = 0;
    for (int r = 0; r < C.nblk[0]; ++r) { C.rows[(size_t)r] = acc; acc += cnt[(size_t)r]; }
  }
  R.data.assign((size_t)off, 0.0);
  for (size_t i = 0; i < Cin.ids.size(); ++i) {
    const size_t pos = (size_t)(std::lower_bound(ids.begin(), ids.end(), Cin.ids[i]) - ids.begin());
    const int64_t sz = Cin.block_size(Cin.ids[i]);
    std::copy(dCin + Cin.offsets[i], dCin + Cin.offsets[i] + sz, R.data.begin() + C.offsets[pos]);
  }
  // pair ranges per result block
  std::vector<int64_t> pstart(ids.size() + 1, 0);
  {
    size_t p = 0;
    for (size_t i = 0; i < ids.size(); ++i) {
      pstart[i] = (int64_t)p;
      while (p < pairs.size() && pairs[p].c == ids[i]) ++p;
    }
    pstart[ids.size()] = (int64_t)pairs.size();
  }
  double flops = 0.0;
  for (const Pair& p : pairs) {
    std::vector<int> da(A.order), db(B.order);
    A.block_dims(A.ids[(size_t)p.a], da.data());
    B.block_dims(B.ids[(size_t)p.b], db.data());
    double mm = 1, nn = 1, kk = 1;
    for (int ax : m.rowA) mm *= da[ax];
    for (int ax : m.colB) nn *= db[ax];
    for (int ax : m.colA) kk *= da[ax];
    flops += 2.0 * mm * nn * kk;
  }
  R.flops = flops;
  R.pairs.clear();
  for (const Pair& p : pairs) R.pairs.push_back({p.c, A.ids[(size_t)p.a], B.ids[(size_t)p.b]});

  const int64_t ncb = (int64_t)ids.size();
#ifdef _OPENMP
  const int nt = nthreads > 0 ? nthreads : omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 1) num_threads(nt)
#endif
  for (int64_t ci = 0; ci < ncb; ++ci) {
    std::vector<int> dc(C.order), da(A.order), db(B.order);
    C.block_dims(ids[(size_t)ci], dc.data());
    double* pc = R.data.data() + C.offsets[(size_t)ci];
    const int64_t csz = C.block_size(ids[(size_t)ci]);
    // beta once per result block
    if (bytes_zero(beta)) {
      for (int64_t e = 0; e < csz; ++e) pc[e] = 0.0;
    } else {
      for (int64_t e = 0; e < csz; ++e) pc[e] = beta * pc[e];
    }
    if (bytes_zero(alpha)) continue;
    std::vector<double> buf;
    for (int64_t p = pstart[(size_t)ci]; p < pstart[(size_t)ci + 1]; ++p) {
      const Pair& pr = pairs[(size_t)p];
      A.block_dims(A.ids[(size_t)pr.a], da.data());
      B.block_dims(B.ids[(size_t)pr.b], db.data());
      const double* pa = dA + A.offsets[(size_t)pr.a];
      const double* pb = dB + B.offsets[(size_t)pr.b];
      if (lapack_blocks) {
        lapack_triple(pa, pb, pc, da.data(), A.order, db.data(), B.order, dc.data(), C.order, m,
                      alpha, 1.0, gemm, rfn, buf);
      } else {
        const auto rA = scatter_of(m.rowA, da.data(), A.order), kA = scatter_of(m.colA, da.data(), A.order);
        const auto kB = scatter_of(m.rowB, db.data(), B.order), cB_ = scatter_of(m.colB, db.data(), B.order);
        const auto rC = scatter_of(m.rowC, dc.data(), C.order), cC = scatter_of(m.colC, dc.data(), C.order);
        xmm_triple<double>(pa, pb, pc, rA, kA, kB, cB_, rC, cC, alpha, 1.0, false);
      }
    }
  }
  R.seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  return true;
}

template <typename T>
int kernel_xmm(const char* expr, int nA, const int* sA, int nB, const int* sB, int nC,
                      const int* sC, T alpha, T beta, const T* a, const T* b, T* c,
                      int64_t nb_ops, char* err, int errlen) {
  Maps m;
  std::string e;
  if (!parse_contraction(expr ? expr : "", nA, sA, nB, sB, nC, sC, m, e)) { set_err(err, errlen, e); return 1; }
  const auto rA = scatter_of(m.rowA, sA, nA), kA = scatter_of(m.colA, sA, nA);
  const auto kB = scatter_of(m.rowB, sB, nB), cB = scatter_of(m.colB, sB, nB);
  const auto rC = scatter_of(m.rowC, sC, nC), cC = scatter_of(m.colC, sC, nC);
  int64_t za = 1, zb = 1, zc = 1;
  for (int i = 0; i < nA; ++i) za *= sA[i];
  for (int i = 0; i < nB; ++i) zb *= sB[i];
  for (int i = 0; i < nC; ++i) zc *= sC[i];
  for (int64_t op = 0; op < nb_ops; ++op)
    xmm_triple<T>(a + op * za, b + op * zb, c + op * zc, rA, kA, kB, cB, rC, cC, alpha, beta, true);
  return 0;
}

}  // namespace ora

// =========================================================================================
// C API
// =========================================================================================
using namespace ora;
using ora::kernel_xmm;

extern "C" {

int ora_contract_info(const char* expr, int nA, const int* sA, int nB, const int* sB, int nC,
                      const int* sC, int* maps, int* counts, char* err, int errlen) {
  Maps m;
  std::string e;
  if (!parse_contraction(expr ? expr : "", nA, sA, nB, sB, nC, sC, m, e)) { set_err(err, errlen, e); return 1; }
  const std::vector<int>* lists[6] = {&m.rowA, &m.colA, &m.rowB, &m.colB, &m.rowC, &m.colC};
  for (int i = 0; i < 6; ++i) {
    counts[i] = (int)lists[i]->size();
    for (size_t j = 0; j < lists[i]->size() && j < 16; ++j) maps[i * 16 + (int)j] = (*lists[i])[j];
  }
  return 0;
}

int ora_scatter(const int* map, int nmap, const int* sizes, int nsizes, int* out) {
  std::vector<int> mv(map, map + nmap);
  const auto v = scatter_of(mv, sizes, nsizes);
  for (size_t i = 0; i < v.size(); ++i) out[i] = (int)v[i];
  return (int)v.size();
}

void ora_reshape_f64(const double* in, const int* sizes, const int* order, int n, double* out) {
  reshape(in, sizes, order, n, out);
}

int ora_kernel_xmm_f64(const char* expr, int nA, const int* sA, int nB, const int* sB, int nC,
                       const int* sC, double alpha, double beta, const double* a,
                       const double* b, double* c, int64_t nb_ops, char* err, int errlen) {
  return kernel_xmm<double>(expr, nA, sA, nB, sB, nC, sC, alpha, beta, a, b, c, nb_ops, err, errlen);
}

int ora_kernel_xmm_f32(const char* expr, int nA, const int* sA, int nB, const int* sB, int nC,
                       const int* sC, float alpha, float beta, const float* a, const float* b,
                       float* c, int64_t nb_ops, char* err, int errlen) {
  return kernel_xmm<float>(expr, nA, sA, nB, sB, nC, sC, alpha, beta, a, b, c, nb_ops, err, errlen);
}

int ora_kernel_lapack_f64(const char* expr, int nA, const int* sA, int nB, const int* sB,
                          int nC, const int* sC, double alpha, double beta, const double* a,
                          const double* b, double* c, int64_t nb_ops, char* err, int errlen) {
  Maps m;
  std::string e;
  if (!parse_contraction(expr ? expr : "", nA, sA, nB, sB, nC, sC, m, e)) { set_err(err, errlen, e); return 1; }
  int64_t za = 1, zb = 1, zc = 1;
  for (int i = 0; i < nA; ++i) za *= sA[i];
  for (int i = 0; i < nB; ++i) zb *= sB[i];
  for (int i = 0; i < nC; ++i) zc *= sC[i];
  std::vector<double> buf;
  for (int64_t op = 0; op < nb_ops; ++op)
    lapack_triple(a + op * za, b + op * zb, c + op * zc, sA, nA, sB, nB, sC, nC, m, alpha, beta,
                  nullptr, nullptr, buf);
  return 0;
}

int ora_reserve(int order, const int* nblk, const int* bsizes, int64_t n, const int* idx,
                int64_t* ids_out, int64_t* offsets_out, int64_t* rows_out, int64_t* nnz_out,
                char* err, int errlen) {
  BTensor t;
  std::string e;
  if (!reserve(order, nblk, bsizes, n, idx, t, e)) { set_err(err, errlen, e); return 1; }
  std::copy(t.ids.begin(), t.ids.end(), ids_out);
  std::copy(t.offsets.begin(), t.offsets.end(), offsets_out);
  std::copy(t.rows.begin(), t.rows.end(), rows_out);
  *nnz_out = t.nnz;
  return 0;
}

double ora_block_norm(const double* data, int64_t n, int norm) { return block_norm(data, n, norm); }

int64_t ora_filter(int order, const int* nblk, const int* bsizes, int64_t nblocks, int64_t* ids,
                   int64_t* offsets, double* data, double eps, int norm, int compress,
                   int64_t* rows_out, int64_t* nnz_out) {
  BTensor t;
  load_tensor(order, nblk, bsizes, nblocks, ids, offsets, t);
  // Tensor::filter marks blocks with norm < eps as -(id)-1 (Tensor.h:346-353).
  for (int64_t b = 0; b < nblocks; ++b) {
    const int64_t sz = t.block_size(ids[b]);
    if (block_norm(data + offsets[b], sz, norm) < eps) ids[b] = -ids[b] - 1;
  }
  if (!compress) { *nnz_out = t.nnz; return nblocks; }
  int64_t w = 0, off = 0;
  for (int64_t b = 0; b < nblocks; ++b) {
    if (ids[b] < 0) continue;
    const int64_t sz = t.block_size(ids[b]);
    std::memmove(data + off, data + offsets[b], (size_t)sz * sizeof(double));
    ids[w] = ids[b];
    offsets[w] = off;
    off += sz;
    ++w;
  }
  std::vector<int64_t> cnt((size_t)nblk[0], 0);
  for (int64_t b = 0; b < w; ++b) cnt[(size_t)(ids[b] % nblk[0])]++;
  int64_t acc = 0;
  for (int r = 0; r < nblk[0]; ++r) { rows_out[r] = acc; acc += cnt[(size_t)r]; }
  *nnz_out = off;
  return w;
}

void* ora_contract_run(const char* expr, double alpha, int oA, const int* nbA, const int* bsA,
                       int64_t nA, const int64_t* idsA, const int64_t* offA, const double* dA,
                       int oB, const int* nbB, const int* bsB, int64_t nB, const int64_t* idsB,
                       const int64_t* offB, const double* dB, double beta, int oC,
                       const int* nbC, const int* bsC, int64_t nC, const int64_t* idsC,
                       const int64_t* offC, const double* dC, double eps, int norm,
                       int lapack_blocks, int nthreads, char* err, int errlen) {
  BTensor A, B, C;
  load_tensor(oA, nbA, bsA, nA, idsA, offA, A);
  load_tensor(oB, nbB, bsB, nB, idsB, offB, B);
  load_tensor(oC, nbC, bsC, nC, idsC, offC, C);
  auto* R = new ContractResult();
  std::string e;
  if (!contract(expr ? expr : "", alpha, A, dA, B, dB, beta, C, dC, eps, norm, lapack_blocks,
                nthreads, nullptr, nullptr, *R, e)) {
    set_err(err, errlen, e);
    delete R;
    return nullptr;
  }
  return R;
}

int64_t ora_result_npairs(void* h) { return (int64_t)static_cast<ContractResult*>(h)->pairs.size(); }
void ora_result_pairs(void* h, int64_t* t) {
  auto* R = static_cast<ContractResult*>(h);
  for (size_t i = 0; i < R->pairs.size(); ++i) { t[3 * i] = R->pairs[i].c; t[3 * i + 1] = R->pairs[i].a; t[3 * i + 2] = R->pairs[i].b; }
}
int64_t ora_result_nblocks(void* h) { return (int64_t)static_cast<ContractResult*>(h)->C.ids.size(); }
int64_t ora_result_nnz(void* h) { return static_cast<ContractResult*>(h)->C.nnz; }
double ora_result_flops(void* h) { return static_cast<ContractResult*>(h)->flops; }
void ora_result_index(void* h, int64_t* ids, int64_t* offsets) {
  auto* R = static_cast<ContractResult*>(h);
  std::copy(R->C.ids.begin(), R->C.ids.end(), ids);
  std::copy(R->C.offsets.begin(), R->C.offsets.end(), offsets);
}
void ora_result_data(void* h, double* data) {
  auto* R = static_cast<ContractResult*>(h);
  std::copy(R->data.begin(), R->data.end(), data);
}
double ora_result_seconds(void* h) { return static_cast<ContractResult*>(h)->seconds; }
void ora_result_free(void* h) { delete static_cast<ContractResult*>(h); }

}  // extern "C"
