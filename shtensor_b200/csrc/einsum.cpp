// einsum.cpp -- expression -> matrix-dimension maps for the contraction kernels.
//
// Follows the mapping of shtensor's compute_contract_info (src/Basics/ContractInfo.h:69-346),
// which the drop-in must reproduce exactly: axes are numbered by first appearance over the
// three index strings; the contracted set is A∩B, the row set A\B, the column set B\A, each
// ordered by axis number; A's rows/cols, B's rows/cols and C's rows/cols are the local mode
// positions of those sets.  The error texts are the reference's.  Two inputs the reference
// mis-maps silently are rejected here: an index count different from the tensor order, and
// an output index list that is not exactly the free indices of A and B.
#include <algorithm>
#include <cctype>
#include <set>

#include "sht_internal.h"

namespace sht {
namespace {

enum class Tok { Indices, Comma, Arrow };

struct Token {
  Tok kind;
  int pos;
  std::string text;
};

std::vector<Token> tokenize(const std::string& s) {
  std::vector<Token> out;
  auto is_index = [](char c) { return std::isalpha(static_cast<unsigned char>(c)) || c == '_'; };
  size_t i = 0;
  while (i < s.size()) {
    const char c = s[i];
    if (std::isspace(static_cast<unsigned char>(c))) { ++i; continue; }
    if (is_index(c)) {
      size_t j = i;
      while (j < s.size() && is_index(s[j])) ++j;
      out.push_back({Tok::Indices, static_cast<int>(i), s.substr(i, j - i)});
      i = j;
    } else if (c == ',') {
      out.push_back({Tok::Comma, static_cast<int>(i), ","});
      ++i;
    } else if (c == '-' && i + 1 < s.size() && s[i + 1] == '>') {
      out.push_back({Tok::Arrow, static_cast<int>(i), "->"});
      i += 2;
    } else {
      fail(SHT_ERR_PARSE, "Unknown character in equation at position " + std::to_string(i) + ": " +
                              std::string(1, c));
    }
  }
  return out;
}

const char* tok_name(Tok t) {
  switch (t) {
    case Tok::Indices: return "index";
    case Tok::Comma: return ",";
    default: return "->";
  }
}

}  // namespace

void parse_einsum(const std::string& expr, int nA, const int* sA, int nB, const int* sB, int nC,
                  const int* sC, ShtMaps& m) {
  if (expr.empty()) fail(SHT_ERR_PARSE, "Equation is empty");
  const std::vector<Token> toks = tokenize(expr);
  static const Tok grammar[5] = {Tok::Indices, Tok::Comma, Tok::Indices, Tok::Arrow, Tok::Indices};
  for (int i = 0; i < 5; ++i) {
    if (i >= static_cast<int>(toks.size()))
      fail(SHT_ERR_PARSE, std::string("Unexpected end of expression, expected ") + tok_name(grammar[i]));
    if (toks[i].kind != grammar[i])
      fail(SHT_ERR_PARSE, std::string("Expected ") + tok_name(grammar[i]) + " at position " +
                              std::to_string(toks[i].pos));
  }
  if (toks.size() != 5) fail(SHT_ERR_PARSE, "Invalid syntax");

  // axis numbering by first appearance
  std::vector<char> seen;
  auto axes_of = [&seen](const std::string& idx) {
    std::vector<int> ax;
    for (char c : idx) {
      auto it = std::find(seen.begin(), seen.end(), c);
      if (it == seen.end()) { seen.push_back(c); it = seen.end() - 1; }
      ax.push_back(static_cast<int>(it - seen.begin()));
    }
    return ax;
  };
  const std::vector<int> a = axes_of(toks[0].text), b = axes_of(toks[2].text), c = axes_of(toks[4].text);
  auto unique_count = [](const std::vector<int>& v) { return std::set<int>(v.begin(), v.end()).size(); };
  if (unique_count(a) != a.size() || unique_count(b) != b.size() || unique_count(c) != c.size())
    fail(SHT_ERR_PARSE, "Duplicate tensor indices");

  auto in = [](const std::vector<int>& v, int x) { return std::find(v.begin(), v.end(), x) != v.end(); };
  std::vector<int> con, free_a, free_b;  // ordered by axis number
  for (int ax = 0; ax < static_cast<int>(seen.size()); ++ax) {
    const bool ia = in(a, ax), ib = in(b, ax);
    if (ia && ib) con.push_back(ax);
    else if (ia) free_a.push_back(ax);
    else if (ib) free_b.push_back(ax);
  }
  if (free_a.empty() || free_b.empty()) fail(SHT_ERR_PARSE, "Element-wise multiplication not supported");
  if (con.empty()) fail(SHT_ERR_PARSE, "No indices found over which to contract");
  if (free_a.size() + free_b.size() != c.size()) fail(SHT_ERR_PARSE, "Dimension mismatch");
  for (int ax : c)
    if (!in(free_a, ax) && !in(free_b, ax))
      fail(SHT_ERR_PARSE, "Output indices must be the free indices of both inputs");
  if (static_cast<int>(a.size()) != nA || static_cast<int>(b.size()) != nB || static_cast<int>(c.size()) != nC)
    fail(SHT_ERR_PARSE, "Number of indices does not match tensor order");
  if (nA > kMaxOrder || nB > kMaxOrder || nC > kMaxOrder)
    fail(SHT_ERR_UNSUPPORTED, "tensor order above " + std::to_string(kMaxOrder));

  auto positions = [](const std::vector<int>& tensor_axes, const std::vector<int>& sel) {
    std::vector<int> out;
    for (int ax : sel) out.push_back(static_cast<int>(std::find(tensor_axes.begin(), tensor_axes.end(), ax) - tensor_axes.begin()));
    return out;
  };
  m.rowA = positions(a, free_a);
  m.colA = positions(a, con);
  m.rowB = positions(b, con);
  m.colB = positions(b, free_b);
  m.rowC = positions(c, free_a);
  m.colC = positions(c, free_b);

  auto check = [](const std::vector<int>& m1, const std::vector<int>& m2, const int* d1, const int* d2,
                  const char* n1, const char* n2) {
    if (!d1 || !d2) return;
    for (size_t i = 0; i < m1.size(); ++i)
      if (d1[m1[i]] != d2[m2[i]])
        fail(SHT_ERR_SIZE, "Sizes for dimensions " + std::to_string(m1[i]) + " in " + n1 +
                               " and for dimension " + std::to_string(m2[i]) + " in " + n2 +
                               " do not match.");
  };
  check(m.rowA, m.rowC, sA, sC, "tensor A", "tensor C");
  check(m.colB, m.colC, sB, sC, "tensor B", "tensor C");
  check(m.colA, m.rowB, sA, sB, "tensor A", "tensor B");
}

}  // namespace sht
