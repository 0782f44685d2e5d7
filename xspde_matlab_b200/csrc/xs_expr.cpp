// MATLAB anonymous-function subset: lexer, parser, device-code generator and
// FP64 host evaluator.  See xs_expr.hpp for the contract.
#include "xs_expr.hpp"

#include <cctype>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <functional>
#include <set>
#include <sstream>

namespace xs {

namespace {

// ----------------------------------------------------------------------------
// Lexer
// ----------------------------------------------------------------------------
enum class TK { End, Num, Ident, Op, LParen, RParen, LBrack, RBrack, LBrace, RBrace, Comma, Semi, At, Field, Colon };

struct Tok {
  TK k;
  std::string s;
  double v = 0;
  bool imag = false;
};

std::vector<Tok> lex(const std::string& src) {
  std::vector<Tok> out;
  size_t i = 0, n = src.size();
  auto prev_allows_transpose = [&]() {
    if (out.empty()) return false;
    const Tok& t = out.back();
    return t.k == TK::Ident || t.k == TK::Num || t.k == TK::RParen || t.k == TK::RBrack ||
           t.k == TK::RBrace || t.k == TK::Field || (t.k == TK::Op && (t.s == "'" || t.s == ".'"));
  };
  while (i < n) {
    char c = src[i];
    if (isspace((unsigned char)c)) { ++i; continue; }
    if (c == '.' && i + 2 < n && src[i + 1] == '.' && src[i + 2] == '.') {  // continuation
      while (i < n && src[i] != '\n') ++i;
      continue;
    }
    if (isdigit((unsigned char)c) || (c == '.' && i + 1 < n && isdigit((unsigned char)src[i + 1]))) {
      size_t j = i;
      while (j < n && isdigit((unsigned char)src[j])) ++j;
      if (j < n && src[j] == '.' && !(j + 1 < n && strchr("*/^\\'", src[j + 1]))) {
        ++j;
        while (j < n && isdigit((unsigned char)src[j])) ++j;
      }
      if (j < n && (src[j] == 'e' || src[j] == 'E')) {
        size_t k = j + 1;
        if (k < n && (src[k] == '+' || src[k] == '-')) ++k;
        if (k < n && isdigit((unsigned char)src[k])) {
          j = k;
          while (j < n && isdigit((unsigned char)src[j])) ++j;
        }
      }
      Tok t{TK::Num, src.substr(i, j - i)};
      t.v = strtod(t.s.c_str(), nullptr);
      if (j < n && (src[j] == 'i' || src[j] == 'j') && !(j + 1 < n && (isalnum((unsigned char)src[j + 1]) || src[j + 1] == '_'))) {
        t.imag = true;
        ++j;
      }
      out.push_back(t);
      i = j;
      continue;
    }
    if (isalpha((unsigned char)c) || c == '_') {
      size_t j = i;
      while (j < n && (isalnum((unsigned char)src[j]) || src[j] == '_')) ++j;
      out.push_back(Tok{TK::Ident, src.substr(i, j - i)});
      i = j;
      continue;
    }
    if (c == '.' && i + 1 < n && (isalpha((unsigned char)src[i + 1]) || src[i + 1] == '_')) {
      size_t j = i + 1;
      while (j < n && (isalnum((unsigned char)src[j]) || src[j] == '_')) ++j;
      out.push_back(Tok{TK::Field, src.substr(i + 1, j - i - 1)});
      i = j;
      continue;
    }
    auto two = src.substr(i, 2);
    if (two == ".*" || two == "./" || two == ".^" || two == ".\\" || two == "<=" || two == ">=" ||
        two == "==" || two == "~=" || two == "&&" || two == "||") {
      out.push_back(Tok{TK::Op, two});
      i += 2;
      continue;
    }
    if (two == ".'") {
      out.push_back(Tok{TK::Op, ".'"});
      i += 2;
      continue;
    }
    switch (c) {
      case '(': out.push_back(Tok{TK::LParen, "("}); break;
      case ')': out.push_back(Tok{TK::RParen, ")"}); break;
      case '[': out.push_back(Tok{TK::LBrack, "["}); break;
      case ']': out.push_back(Tok{TK::RBrack, "]"}); break;
      case '{': out.push_back(Tok{TK::LBrace, "{"}); break;
      case '}': out.push_back(Tok{TK::RBrace, "}"}); break;
      case ',': out.push_back(Tok{TK::Comma, ","}); break;
      case ';': out.push_back(Tok{TK::Semi, ";"}); break;
      case '@': out.push_back(Tok{TK::At, "@"}); break;
      case ':': out.push_back(Tok{TK::Colon, ":"}); break;
      case '\'':
        if (prev_allows_transpose()) {
          out.push_back(Tok{TK::Op, "'"});
          break;
        }
        throw GrammarError("strings are not supported in xSPDE device functions");
      case '+': case '-': case '*': case '/': case '^': case '\\': case '<': case '>': case '~': case '&': case '|':
        out.push_back(Tok{TK::Op, std::string(1, c)});
        break;
      default:
        throw GrammarError(std::string("unexpected character '") + c + "'");
    }
    ++i;
  }
  out.push_back(Tok{TK::End, ""});
  return out;
}

// ----------------------------------------------------------------------------
// Parser (MATLAB precedence: || && | & comparisons : +- */ unary ^ postfix)
// ----------------------------------------------------------------------------
struct Parser {
  std::vector<Tok> t;
  size_t p = 0;
  int bracket_depth = 0;

  const Tok& cur() const { return t[p]; }
  bool is_op(const char* s) const { return cur().k == TK::Op && cur().s == s; }
  void expect(TK k, const char* what) {
    if (cur().k != k) throw GrammarError(std::string("expected ") + what + " near '" + cur().s + "'");
    ++p;
  }
  static NodeP mk(NK k, const std::string& name = "") {
    auto n = std::make_shared<Node>();
    n->kind = k;
    n->name = name;
    return n;
  }
  NodeP bin(const std::string& op, NodeP l, NodeP r) {
    auto n = mk(NK::Bin, op);
    n->kids = {l, r};
    return n;
  }

  NodeP expr() { return oror(); }
  NodeP oror() {
    auto l = andand();
    while (is_op("||") || is_op("|")) { std::string o = cur().s; ++p; l = bin(o, l, andand()); }
    return l;
  }
  NodeP andand() {
    auto l = cmp();
    while (is_op("&&") || is_op("&")) { std::string o = cur().s; ++p; l = bin(o, l, cmp()); }
    return l;
  }
  NodeP cmp() {
    auto l = add();
    while (is_op("<") || is_op(">") || is_op("<=") || is_op(">=") || is_op("==") || is_op("~=")) {
      std::string o = cur().s;
      ++p;
      l = bin(o, l, add());
    }
    return l;
  }
  bool plus_minus_is_binary() const {
    // Inside [] a space-separated sign starts a new element in MATLAB; we do
    // not support horizontal concatenation, so always treat as binary.
    return true;
  }
  NodeP add() {
    auto l = mul();
    while ((is_op("+") || is_op("-")) && plus_minus_is_binary()) {
      std::string o = cur().s;
      ++p;
      l = bin(o, l, mul());
    }
    return l;
  }
  NodeP mul() {
    auto l = unary();
    while (is_op("*") || is_op("/") || is_op(".*") || is_op("./") || is_op("\\") || is_op(".\\")) {
      std::string o = cur().s;
      ++p;
      l = bin(o, l, unary());
    }
    return l;
  }
  NodeP unary() {
    if (is_op("-") || is_op("+") || is_op("~")) {
      std::string o = cur().s;
      ++p;
      auto n = mk(NK::Un, o);
      n->kids = {unary()};
      return n;
    }
    return power();
  }
  NodeP power() {
    auto l = postfix();
    while (is_op("^") || is_op(".^")) {
      std::string o = cur().s;
      ++p;
      NodeP r;
      if (is_op("-") || is_op("+")) {  // 2^-1
        std::string u = cur().s;
        ++p;
        auto n = mk(NK::Un, u);
        n->kids = {postfix()};
        r = n;
      } else {
        r = postfix();
      }
      l = bin(o, l, r);
    }
    return l;
  }
  std::vector<NodeP> args(TK close) {
    std::vector<NodeP> a;
    if (cur().k == close) { ++p; return a; }
    while (true) {
      if (cur().k == TK::Colon) {
        ++p;
        a.push_back(mk(NK::Colon));
      } else {
        a.push_back(expr());
      }
      if (cur().k == TK::Comma) { ++p; continue; }
      if (cur().k == close) { ++p; break; }
      throw GrammarError("expected ',' or closing bracket near '" + cur().s + "'");
    }
    return a;
  }
  NodeP postfix() {
    auto n = primary();
    while (true) {
      if (cur().k == TK::LParen) {
        ++p;
        auto c = mk(NK::Index);
        c->kids.push_back(n);
        for (auto& a : args(TK::RParen)) c->kids.push_back(a);
        n = c;
      } else if (cur().k == TK::LBrace) {
        ++p;
        auto c = mk(NK::CellIndex);
        c->kids.push_back(n);
        for (auto& a : args(TK::RBrace)) c->kids.push_back(a);
        n = c;
      } else if (cur().k == TK::Field) {
        auto f = mk(NK::Field, cur().s);
        f->kids.push_back(n);
        ++p;
        n = f;
      } else if (is_op("'") || is_op(".'")) {
        auto u = mk(NK::Un, cur().s);
        ++p;
        u->kids = {n};
        n = u;
      } else {
        break;
      }
    }
    return n;
  }
  NodeP primary() {
    const Tok& k = cur();
    if (k.k == TK::Num) {
      auto n = mk(k.imag ? NK::Imag : NK::Num);
      n->num = k.v;
      ++p;
      return n;
    }
    if (k.k == TK::Ident) {
      auto n = mk(NK::Var, k.s);
      ++p;
      return n;
    }
    if (k.k == TK::LParen) {
      ++p;
      auto e = expr();
      expect(TK::RParen, "')'");
      return e;
    }
    if (k.k == TK::LBrack) {
      ++p;
      auto c = mk(NK::Concat);
      std::vector<NodeP> row;
      if (cur().k == TK::RBrack) { ++p; return c; }
      while (true) {
        row.push_back(expr());
        if (cur().k == TK::Comma) { ++p; continue; }
        if (cur().k == TK::Semi) { ++p; c->rows.push_back(row); row.clear(); continue; }
        if (cur().k == TK::RBrack) { ++p; c->rows.push_back(row); break; }
        // MATLAB allows whitespace-separated row elements: "[0 1 1]"
        row.push_back(expr());
        if (cur().k == TK::RBrack) { ++p; c->rows.push_back(row); break; }
        if (cur().k == TK::Semi) { ++p; c->rows.push_back(row); row.clear(); continue; }
        if (cur().k == TK::Comma) { ++p; continue; }
        throw GrammarError("malformed [...] near '" + cur().s + "'");
      }
      return c;
    }
    throw GrammarError("unexpected token '" + k.s + "'");
  }
};

}  // namespace

AnonFn parse_anon(const std::string& text) {
  AnonFn fn;
  fn.text = text;
  Parser ps;
  ps.t = lex(text);
  if (ps.cur().k == TK::At) {
    ++ps.p;
    ps.expect(TK::LParen, "'(' after '@'");
    while (ps.cur().k != TK::RParen) {
      if (ps.cur().k == TK::Ident) fn.params.push_back(ps.cur().s);
      else if (ps.cur().k == TK::Op && ps.cur().s == "~") fn.params.push_back("~");
      else throw GrammarError("bad anonymous-function argument list");
      ++ps.p;
      if (ps.cur().k == TK::Comma) ++ps.p;
    }
    ++ps.p;
  }
  fn.body = ps.expr();
  if (ps.cur().k != TK::End) throw GrammarError("unexpected trailing text near '" + ps.cur().s + "'");
  return fn;
}

// ----------------------------------------------------------------------------
// FP64 evaluator (constant folding and the host-side linear operator)
// ----------------------------------------------------------------------------
namespace {

using C = std::complex<double>;
using Vec = std::vector<C>;

struct NotConst {};

struct EvalEnv {
  std::function<bool(const std::string&, Vec&)> var;     // bare identifiers
  std::function<bool(const std::string&, Vec&)> field;   // p.<name>
  std::function<bool(const std::string&, int, Vec&)> cell;  // p.<name>{d}
  std::string pname = "p";
};

Vec bcast(const Vec& a, size_t n) {
  if (a.size() == n) return a;
  if (a.size() == 1) return Vec(n, a[0]);
  throw GrammarError("component count mismatch");
}

C cpow(C a, C b) {
  if (b.imag() == 0 && b.real() == std::floor(b.real()) && std::fabs(b.real()) <= 64) {
    int e = (int)b.real();
    C r = 1;
    C base = e < 0 ? 1.0 / a : a;
    for (int i = 0; i < std::abs(e); ++i) r *= base;
    return r;
  }
  if (a == C(0)) return b.real() > 0 ? C(0) : C(INFINITY);
  return std::exp(b * std::log(a));
}

C apply1(const std::string& f, C z) {
  if (f == "conj") return std::conj(z);
  if (f == "real") return z.real();
  if (f == "imag") return z.imag();
  if (f == "abs") return std::abs(z);
  if (f == "angle") return std::arg(z);
  if (f == "exp") return std::exp(z);
  if (f == "log") return std::log(z);
  if (f == "sqrt") return std::sqrt(z);
  if (f == "sin") return std::sin(z);
  if (f == "cos") return std::cos(z);
  if (f == "tan") return std::tan(z);
  if (f == "sinh") return std::sinh(z);
  if (f == "cosh") return std::cosh(z);
  if (f == "tanh") return std::tanh(z);
  if (f == "sech") return 1.0 / std::cosh(z);
  if (f == "csch") return 1.0 / std::sinh(z);
  if (f == "sec") return 1.0 / std::cos(z);
  if (f == "csc") return 1.0 / std::sin(z);
  if (f == "cot") return 1.0 / std::tan(z);
  if (f == "coth") return 1.0 / std::tanh(z);
  if (f == "asin") return std::asin(z);
  if (f == "acos") return std::acos(z);
  if (f == "atan") return std::atan(z);
  if (f == "sign") return z == C(0) ? C(0) : (z.imag() == 0 ? C(z.real() > 0 ? 1 : -1) : z / std::abs(z));
  if (f == "floor") return C(std::floor(z.real()), std::floor(z.imag()));
  if (f == "ceil") return C(std::ceil(z.real()), std::ceil(z.imag()));
  if (f == "round") return C(std::round(z.real()), std::round(z.imag()));
  if (f == "fix") return C(std::trunc(z.real()), std::trunc(z.imag()));
  if (f == "erf") return std::erf(z.real());
  throw GrammarError("unsupported function '" + f + "'");
}

const std::set<std::string>& unary_funcs() {
  static const std::set<std::string> s = {"conj", "real", "imag", "abs", "angle", "exp", "log", "sqrt", "sin",
                                          "cos", "tan", "sinh", "cosh", "tanh", "sech", "csch", "sec", "csc",
                                          "cot", "coth", "asin", "acos", "atan", "sign", "floor", "ceil",
                                          "round", "fix", "erf"};
  return s;
}

Vec eval(const NodeP& n, const EvalEnv& env);

Vec eval_bin(const std::string& op, const Vec& a, const Vec& b) {
  size_t L = std::max(a.size(), b.size());
  if (a.size() != b.size() && a.size() != 1 && b.size() != 1) throw GrammarError("component count mismatch in '" + op + "'");
  Vec A = bcast(a, L), B = bcast(b, L), R(L);
  for (size_t i = 0; i < L; ++i) {
    C x = A[i], y = B[i];
    if (op == "+") R[i] = x + y;
    else if (op == "-") R[i] = x - y;
    else if (op == "*" || op == ".*") R[i] = x * y;
    else if (op == "/" || op == "./") R[i] = x / y;
    else if (op == "\\" || op == ".\\") R[i] = y / x;
    else if (op == "^" || op == ".^") R[i] = cpow(x, y);
    else if (op == "<") R[i] = x.real() < y.real();
    else if (op == ">") R[i] = x.real() > y.real();
    else if (op == "<=") R[i] = x.real() <= y.real();
    else if (op == ">=") R[i] = x.real() >= y.real();
    else if (op == "==") R[i] = x == y;
    else if (op == "~=") R[i] = x != y;
    else if (op == "&" || op == "&&") R[i] = (x != C(0)) && (y != C(0));
    else if (op == "|" || op == "||") R[i] = (x != C(0)) || (y != C(0));
    else throw GrammarError("unsupported operator " + op);
  }
  if ((op == "*" || op == "/") && a.size() > 1 && b.size() > 1)
    throw GrammarError("matrix '" + op + "' between vectors; use '." + op.substr(0) + "'");
  return R;
}

Vec eval(const NodeP& n, const EvalEnv& env) {
  switch (n->kind) {
    case NK::Num: return {C(n->num)};
    case NK::Imag: return {C(0, n->num)};
    case NK::Var: {
      Vec v;
      if (env.var && env.var(n->name, v)) return v;
      if (n->name == "pi") return {C(M_PI)};
      if (n->name == "i" || n->name == "j") return {C(0, 1)};
      if (n->name == "Inf" || n->name == "inf") return {C(INFINITY)};
      if (n->name == "eps") return {C(2.220446049250313e-16)};
      throw NotConst();
    }
    case NK::Field: {
      if (n->kids[0]->kind != NK::Var || n->kids[0]->name != env.pname) throw GrammarError("field access on non-parameter");
      Vec v;
      if (env.field && env.field(n->name, v)) return v;
      throw NotConst();
    }
    case NK::CellIndex: {
      auto base = n->kids[0];
      if (base->kind != NK::Field || n->kids.size() != 2) throw GrammarError("unsupported {} indexing");
      Vec d = eval(n->kids[1], EvalEnv{});
      Vec v;
      if (env.cell && env.cell(base->name, (int)d[0].real(), v)) return v;
      throw NotConst();
    }
    case NK::Un: {
      Vec a = eval(n->kids[0], env);
      if (n->name == "-") for (auto& x : a) x = -x;
      else if (n->name == "~") for (auto& x : a) x = (x == C(0)) ? 1.0 : 0.0;
      else if (n->name == "'") for (auto& x : a) x = std::conj(x);
      return a;
    }
    case NK::Bin: return eval_bin(n->name, eval(n->kids[0], env), eval(n->kids[1], env));
    case NK::Concat: {
      Vec r;
      for (auto& row : n->rows)
        for (auto& e : row) {
          Vec v = eval(e, env);
          r.insert(r.end(), v.begin(), v.end());
        }
      return r;
    }
    case NK::Index: {
      auto base = n->kids[0];
      if (base->kind == NK::Var && unary_funcs().count(base->name) && n->kids.size() == 2) {
        Vec a = eval(n->kids[1], env);
        for (auto& x : a) x = apply1(base->name, x);
        return a;
      }
      if (base->kind == NK::Var && (base->name == "atan2" || base->name == "min" || base->name == "max" ||
                                    base->name == "mod" || base->name == "rem") && n->kids.size() == 3) {
        Vec a = eval(n->kids[1], env), b = eval(n->kids[2], env);
        size_t L = std::max(a.size(), b.size());
        a = bcast(a, L);
        b = bcast(b, L);
        Vec r(L);
        for (size_t i = 0; i < L; ++i) {
          double x = a[i].real(), y = b[i].real();
          if (base->name == "atan2") r[i] = std::atan2(x, y);
          else if (base->name == "min") r[i] = std::min(x, y);
          else if (base->name == "max") r[i] = std::max(x, y);
          else if (base->name == "mod") r[i] = y == 0 ? x : x - std::floor(x / y) * y;
          else r[i] = y == 0 ? x : x - std::trunc(x / y) * y;
        }
        return r;
      }
      // indexing a vector-valued parameter: p.dx(2), p.ranges(1)
      Vec b = eval(base, env);
      if (n->kids.size() == 2 && n->kids[1]->kind != NK::Colon) {
        Vec idx = eval(n->kids[1], EvalEnv{});
        Vec r;
        for (auto& k : idx) {
          int ii = (int)k.real();
          if (ii < 1 || ii > (int)b.size()) throw GrammarError("index out of range");
          r.push_back(b[ii - 1]);
        }
        return r;
      }
      throw NotConst();
    }
    case NK::Colon: throw NotConst();
  }
  throw NotConst();
}

// ----------------------------------------------------------------------------
// Device-code generator
// ----------------------------------------------------------------------------
struct Val {
  int len = 1;
  bool cplx = false;
  bool imag = false;                    // purely imaginary: c[] are real expressions of the imaginary part
  bool spatial = false;                 // depends on the site (a, w, v, x, y, z)
  std::vector<std::string> c;           // per-component C expression (temp names / literals)
};

std::string lit(double v) {
  char buf[64];
  if (std::isinf(v)) return v > 0 ? "(real)INFINITY" : "(real)(-INFINITY)";
  if (std::isnan(v)) return "(real)NAN";
  snprintf(buf, sizeof buf, "(real)(%.17g)", v);
  return buf;
}

struct Gen {
  const GenCtx& ctx;
  std::ostringstream os;
  int ntmp = 0;
  std::map<std::string, std::string> memo;  // expression text -> temp
  std::vector<Reduction>* reds = nullptr;
  std::string pname = "p", aname, wname, vname, kname, kvname, xname;
  std::vector<std::string> aux_names;
  bool in_integrand = false;
  bool stencil = false;  // D1/D2 used: the code reads neighbours through xs_fd1/xs_fd2

  explicit Gen(const GenCtx& c) : ctx(c) {}

  std::string tmp(bool cplx, const std::string& expr) {
    auto key = std::string(cplx ? "c:" : "r:") + expr;
    auto it = memo.find(key);
    if (it != memo.end()) return it->second;
    std::string name = "t" + std::to_string(ntmp++);
    os << "  const " << (cplx ? "cx " : "real ") << name << " = " << expr << ";\n";
    memo[key] = name;
    return name;
  }

  Val constant(const Vec& v, bool allow_imag = false) {
    Val r;
    r.len = (int)v.size();
    r.cplx = false;
    for (auto& z : v)
      if (z.imag() != 0) r.cplx = true;
    if (allow_imag && r.cplx) {
      bool pure = true;
      for (auto& z : v) pure = pure && z.real() == 0;
      if (pure) {  // e.g. 0.5i: kept as its imaginary part
        r.cplx = false;
        r.imag = true;
        for (auto& z : v) r.c.push_back(lit(z.imag()));
        return r;
      }
    }
    for (auto& z : v) r.c.push_back(r.cplx ? "mkcx(" + lit(z.real()) + "," + lit(z.imag()) + ")" : lit(z.real()));
    return r;
  }

  EvalEnv const_env() const {
    EvalEnv e;
    e.pname = pname;
    const GenCtx* c = &ctx;
    e.field = [c](const std::string& f, Vec& out) {
      auto vec = [&](const std::vector<double>& x) {
        out.clear();
        for (double d : x) out.push_back(C(d));
        return true;
      };
      if (f == "dx") return vec(c->dx);
      if (f == "dk") return vec(c->dk);
      if (f == "origins") return vec(c->origins);
      if (f == "ranges") return vec(c->ranges);
      if (f == "dt") { out = {C(c->dt)}; return true; }
      if (c->runtime)
        for (auto& r : *c->runtime)
          if (r == f) return false;  // a per-instance value: not a compile-time constant
      if (c->scalars) {
        auto it = c->scalars->values.find(f);
        if (it != c->scalars->values.end()) { out = {C(it->second)}; return true; }
      }
      return false;
    };
    return e;
  }

  bool try_const(const NodeP& n, Vec& v) {
    try {
      v = eval(n, const_env());
      return true;
    } catch (const NotConst&) {
      return false;
    }
  }

  Val var(const std::string& name) {
    Val r;
    if (name == aname && !aname.empty()) {
      r.len = ctx.nfield;
      r.cplx = true;
      r.spatial = true;
      for (int i = 0; i < ctx.nfield; ++i) r.c.push_back("a[" + std::to_string(i) + "]");
      return r;
    }
    if (name == wname && !wname.empty()) {
      if (ctx.nnoise <= 0) {  // no noise cell: the argument is the scalar 0 (xnoise.m:27, w{1} = 0)
        r.c = {"(real)0"};
        return r;
      }
      r.len = ctx.nnoise;
      r.spatial = true;
      for (int i = 0; i < ctx.nnoise; ++i) r.c.push_back("w[" + std::to_string(i) + "]");
      return r;
    }
    if (name == xname && !xname.empty()) {  // auxiliary cell (p.define, xpath.m:36-45): complex
      r.len = ctx.naux;
      r.cplx = true;
      r.spatial = true;
      for (int i = 0; i < ctx.naux; ++i) r.c.push_back("xa[" + std::to_string(i) + "]");
      return r;
    }
    if (name == kname && !kname.empty()) {  // k-filtered noise cell (xnoise.m:39-50): complex
      r.len = ctx.nknoise;
      r.cplx = true;
      r.spatial = true;
      for (int i = 0; i < ctx.nknoise; ++i) r.c.push_back("zk[" + std::to_string(i) + "]");
      return r;
    }
    if (name == kvname && !kvname.empty()) {  // k-filtered randoms (xrandom.m:24-29): complex
      r.len = ctx.nkrand;
      r.cplx = true;
      r.spatial = true;
      for (int i = 0; i < ctx.nkrand; ++i) r.c.push_back("vk[" + std::to_string(i) + "]");
      return r;
    }
    if (name == vname && !vname.empty()) {
      if (ctx.nrand <= 0) {  // no random cell: the argument is the scalar 0 (xrandom.m, w{1} = 0)
        r.c = {"(real)0"};
        return r;
      }
      r.len = ctx.nrand;
      r.spatial = true;
      for (int i = 0; i < ctx.nrand; ++i) r.c.push_back("v[" + std::to_string(i) + "]");
      return r;
    }
    throw GrammarError("unknown identifier '" + name + "'");
  }

  Val coord(int d) {  // d: 0 = t, 1 = x, 2 = y, 3 = z
    Val r;
    if (d == 0) { r.c = {"t"}; return r; }
    if (d > ctx.ndim) throw GrammarError("space dimension " + std::to_string(d) + " is not present");
    static const char* nm[] = {"t", "x", "y", "z"};
    r.spatial = true;
    r.c = {nm[d]};
    return r;
  }

  Val field(const std::string& f) {
    if (f == "t") return coord(0);
    if (f == "x") return coord(1);
    if (f == "y") return coord(2);
    if (f == "z") return coord(3);
    if (ctx.kgrid && (f == "kx" || f == "ky" || f == "kz")) {
      const int d = f == "kx" ? 1 : (f == "ky" ? 2 : 3);
      if (d > ctx.ndim) throw GrammarError("space dimension of 'p." + f + "' is not present");
      static const char* ix[] = {"", "i1", "i2", "i3"};
      Val r;
      r.spatial = true;
      r.c = {"((real)xs_kt" + std::to_string(d) + "[" + ix[d] + "])"};
      return r;
    }
    if (f == "Dx" || f == "Dy" || f == "Dz" || f == "kx" || f == "ky" || f == "kz" || f == "D" || f == "k")
      throw GrammarError("k-space grid 'p." + f + "' is only available in p.linear and observe");
    if (ctx.runtime)
      for (size_t k = 0; k < ctx.runtime->size(); ++k)
        if ((*ctx.runtime)[k] == f) {
          Val r;
          r.c = {"((real)prm[" + std::to_string(k) + "])"};
          return r;
        }
    Vec v;
    auto e = const_env();
    if (e.field(f, v)) return constant(v);
    throw GrammarError("unknown parameter 'p." + f + "' (pass it as a named scalar)");
  }

  static std::string fname(const std::string& f) { return "xs_" + f; }

  Val un(const std::string& op, const Val& a) {
    Val r = a;
    r.c.clear();
    for (auto& x : a.c) {
      if (op == "-") r.c.push_back(tmp(a.cplx, "-" + x));
      else if (op == "+") r.c.push_back(x);
      else if (op == "~") { r.cplx = false; r.c.push_back(tmp(false, "xs_not(" + x + ")")); }
      else if (op == "'" ) r.c.push_back(a.cplx ? tmp(true, "xs_conj(" + x + ")") : x);
      else if (op == ".'") r.c.push_back(x);
    }
    return r;
  }

  // A purely imaginary value as an ordinary complex one.
  Val mat(const Val& v) {
    if (!v.imag) return v;
    Val r = v;
    r.imag = false;
    r.cplx = true;
    for (auto& c : r.c) c = tmp(true, "mkcx((real)0, " + c + ")");
    return r;
  }

  // + - * / with a purely imaginary operand (i b): the forms below are what the
  // full complex arithmetic (prelude operators, Smith's division) computes for
  // finite operands, without the products and sums with the zero real part.
  bool imag_bin(const std::string& op, const Val& a, const Val& b, Val& r) {
    const bool mul = op == "*" || op == ".*", dv = op == "/" || op == "./", add = op == "+", sub = op == "-";
    if (!(mul || dv || add || sub)) return false;
    if (mul && op == "*" && a.len > 1 && b.len > 1) return false;
    auto kind = [](const Val& v) { return v.imag ? 'i' : (v.cplx ? 'c' : 'r'); };
    const char ka = kind(a), kb = kind(b);
    r.len = std::max(a.len, b.len);
    r.spatial = a.spatial || b.spatial;
    r.c.clear();
    for (int i = 0; i < r.len; ++i) {
      const std::string x = "(" + a.c[a.len == 1 ? 0 : i] + ")", y = "(" + b.c[b.len == 1 ? 0 : i] + ")";
      char out;
      std::string e;
      if (ka == 'i' && kb == 'r') {
        if (mul) { out = 'i'; e = x + " * " + y; }
        else if (dv) { out = 'i'; e = x + " / " + y; }
        else { out = 'c'; e = "mkcx(" + std::string(add ? "" : "-") + y + ", " + x + ")"; }
      } else if (ka == 'r' && kb == 'i') {
        if (mul) { out = 'i'; e = x + " * " + y; }
        else if (dv) { out = 'i'; e = "-(" + x + " / " + y + ")"; }
        else { out = 'c'; e = "mkcx(" + x + ", " + (add ? "" : "-") + y + ")"; }
      } else if (ka == 'i' && kb == 'i') {
        if (mul) { out = 'r'; e = "-(" + x + " * " + y + ")"; }
        else if (dv) { out = 'r'; e = x + " / " + y; }
        else { out = 'i'; e = x + (add ? " + " : " - ") + y; }
      } else if (ka == 'i' && kb == 'c') {
        if (mul) { out = 'c'; e = "mkcx(-(" + x + " * " + y + ".im), " + x + " * " + y + ".re)"; }
        else if (dv) return false;
        else if (add) { out = 'c'; e = "mkcx(" + y + ".re, " + x + " + " + y + ".im)"; }
        else { out = 'c'; e = "mkcx(-" + y + ".re, " + x + " - " + y + ".im)"; }
      } else if (ka == 'c' && kb == 'i') {
        if (mul) { out = 'c'; e = "mkcx(-(" + x + ".im * " + y + "), " + x + ".re * " + y + ")"; }
        else if (dv) { out = 'c'; e = "mkcx(" + x + ".im / " + y + ", -(" + x + ".re / " + y + "))"; }
        else { out = 'c'; e = "mkcx(" + x + ".re, " + x + ".im " + (add ? "+ " : "- ") + y + ")"; }
      } else {
        return false;
      }
      if (i == 0) {
        r.imag = out == 'i';
        r.cplx = out == 'c';
      } else if ((out == 'i') != r.imag || (out == 'c') != r.cplx) {
        return false;
      }
      r.c.push_back(tmp(out == 'c', e));
    }
    return true;
  }

  Val bin(const std::string& op, const Val& a0, const Val& b0, const NodeP& rnode) {
    if (a0.len != b0.len && a0.len != 1 && b0.len != 1)
      throw GrammarError("component count mismatch (" + std::to_string(a0.len) + " vs " + std::to_string(b0.len) + ") in '" + op + "'");
    if (a0.imag || b0.imag) {
      Val ri;
      if (imag_bin(op, a0, b0, ri)) return ri;
    }
    const Val a = mat(a0), b = mat(b0);
    if ((op == "*" || op == "/") && a.len > 1 && b.len > 1)
      throw GrammarError("matrix '" + op + "' between vectors; use '." + op + "'");
    Val r;
    r.len = std::max(a.len, b.len);
    r.spatial = a.spatial || b.spatial;
    bool cmp = op == "<" || op == ">" || op == "<=" || op == ">=" || op == "==" || op == "~=" ||
               op == "&" || op == "&&" || op == "|" || op == "||";
    // integer power -> repeated multiplication
    Vec ev;
    bool ipow = false;
    int ie = 0;
    if ((op == ".^" || op == "^") && try_const(rnode, ev) && ev.size() == 1 && ev[0].imag() == 0 &&
        ev[0].real() == std::floor(ev[0].real()) && std::fabs(ev[0].real()) <= 16) {
      ipow = true;
      ie = (int)ev[0].real();
    }
    bool cplx = a.cplx || b.cplx;
    if (op == ".^" || op == "^") {
      if (!ipow) cplx = true;  // real^nonint is complex for negative bases in MATLAB
      else cplx = a.cplx;
    }
    if (cmp) cplx = false;
    r.cplx = cplx;
    // division by a real literal constant: multiply by its reciprocal (within one rounding of the
    // quotient; the divide is several instructions, the multiply one)
    std::string recip;
    if ((op == "/" || op == "./") && !b.cplx) {
      Vec cv;
      if (try_const(rnode, cv) && cv.size() == 1 && cv[0].imag() == 0 && cv[0].real() != 0 &&
          std::isfinite(cv[0].real()) && std::isfinite(1.0 / cv[0].real())) {
        char buf[64];
        snprintf(buf, sizeof buf, "(real)(%.17g)", 1.0 / cv[0].real());
        recip = buf;
      }
    }
    for (int i = 0; i < r.len; ++i) {
      const std::string& x = a.c[a.len == 1 ? 0 : i];
      const std::string& y = b.c[b.len == 1 ? 0 : i];
      std::string e;
      if (op == "+" || op == "-") e = x + " " + op + " " + y;
      else if (op == "*" || op == ".*") e = x + " * " + y;
      else if (op == "/" || op == "./") e = recip.empty() ? x + " / " + y : x + " * " + recip;
      else if (op == "\\" || op == ".\\") e = y + " / " + x;
      else if (op == "^" || op == ".^") {
        if (ipow) e = "xs_powi<" + std::to_string(ie) + ">(" + x + ")";
        else e = "xs_pow(" + x + ", " + y + ")";
      } else if (op == "<") e = "xs_lt(" + x + ", " + y + ")";
      else if (op == ">") e = "xs_lt(" + y + ", " + x + ")";
      else if (op == "<=") e = "xs_le(" + x + ", " + y + ")";
      else if (op == ">=") e = "xs_le(" + y + ", " + x + ")";
      else if (op == "==") e = "xs_eq(" + x + ", " + y + ")";
      else if (op == "~=") e = "((real)1 - xs_eq(" + x + ", " + y + "))";
      else if (op == "&" || op == "&&") e = "xs_and(" + x + ", " + y + ")";
      else if (op == "|" || op == "||") e = "xs_or(" + x + ", " + y + ")";
      else throw GrammarError("unsupported operator '" + op + "'");
      r.c.push_back(tmp(cplx, e));
    }
    return r;
  }

  bool is_conj_of(const NodeP& c, const NodeP& x) {
    if (c->kind != NK::Index || c->kids.size() != 2 || c->kids[0]->kind != NK::Var || c->kids[0]->name != "conj") return false;
    return same(c->kids[1], x);
  }
  static bool same(const NodeP& a, const NodeP& b) {
    if (a->kind != b->kind || a->name != b->name || a->num != b->num || a->kids.size() != b->kids.size()) return false;
    for (size_t i = 0; i < a->kids.size(); ++i)
      if (!same(a->kids[i], b->kids[i])) return false;
    if (a->rows.size() != b->rows.size()) return false;
    return true;
  }

  Val gen(const NodeP& n) { return mat(gen_raw(n)); }

  // sv * n for a scale sv that does not depend on the site (the step h times literal factors;
  // real, purely imaginary or complex), with the scale pushed through sums, negations and
  // quotients, literal factors folded into it and the rest applied to one scalar (real or purely
  // imaginary) factor of each product, so that an accumulation c0 + sv*n contracts into fused
  // multiply-adds.  Anything else is multiplied by the scale.
  Val gen_h(const NodeP& n, const Val& sv) {
    Vec cv;
    if (n->kind != NK::Colon && try_const(n, cv)) return bin("*", sv, constant(cv, true), nullptr);
    if (n->kind == NK::Bin && (n->name == "+" || n->name == "-") && n->kids.size() == 2)
      return bin(n->name, gen_h(n->kids[0], sv), gen_h(n->kids[1], sv), nullptr);
    if (n->kind == NK::Un && n->name == "-" && n->kids.size() == 1) return un("-", gen_h(n->kids[0], sv));
    if (n->kind == NK::Un && n->name == "+" && n->kids.size() == 1) return gen_h(n->kids[0], sv);
    if (n->kind == NK::Bin && (n->name == "*" || n->name == ".*") && n->kids.size() == 2) {
      const NodeP &ln = n->kids[0], &rn = n->kids[1];
      Vec lc, rc;
      const bool lk = try_const(ln, lc) && lc.size() == 1, rk = try_const(rn, rc) && rc.size() == 1;
      if (lk) return gen_h(rn, bin("*", sv, constant(lc, true), nullptr));
      if (rk) return gen_h(ln, bin("*", sv, constant(rc, true), nullptr));
      const Val l = gen_raw(ln), r = gen_raw(rn);
      auto scalar = [](const Val& v) { return v.len == 1 && !v.cplx; };
      if (scalar(l)) return bin(n->name, gen_h(ln, sv), r, rn);
      if (scalar(r)) return bin(n->name, l, gen_h(rn, sv), rn);
    }
    if (n->kind == NK::Bin && (n->name == "/" || n->name == "./") && n->kids.size() == 2) {
      Vec dc;
      if (try_const(n->kids[1], dc) && dc.size() == 1 && dc[0] != C(0.0) && std::isfinite(std::abs(1.0 / dc[0])))
        return gen_h(n->kids[0], bin("*", sv, constant({C(1.0) / dc[0]}, true), nullptr));
      return bin(n->name, gen_h(n->kids[0], sv), gen_raw(n->kids[1]), n->kids[1]);
    }
    return bin("*", sv, gen_raw(n), nullptr);
  }

  // gen() that may return a purely imaginary value (consumed only by bin()).
  Val gen_raw(const NodeP& n) {
    Vec cv;
    if (n->kind != NK::Colon && try_const(n, cv)) return constant(cv, true);
    switch (n->kind) {
      case NK::Num: case NK::Imag: return constant(eval(n, EvalEnv{}));
      case NK::Var: return var(n->name);
      case NK::Field: {
        if (n->kids[0]->kind != NK::Var || n->kids[0]->name != pname) throw GrammarError("field access on a non-parameter");
        return field(n->name);
      }
      case NK::CellIndex: {
        auto base = n->kids[0];
        if (base->kind == NK::Field && base->name == "r" && n->kids.size() == 2) {
          Vec d;
          if (!try_const(n->kids[1], d)) throw GrammarError("p.r{d} needs a constant d");
          return coord((int)d[0].real() - 1);
        }
        throw GrammarError("unsupported cell indexing");
      }
      case NK::Un: return un(n->name, gen(n->kids[0]));
      case NK::Bin: {
        // abs(x).^2 and abs(x)^2 -> |x|^2 without the square root
        if ((n->name == ".^" || n->name == "^") && n->kids[0]->kind == NK::Index && n->kids[0]->kids.size() == 2 &&
            n->kids[0]->kids[0]->kind == NK::Var && n->kids[0]->kids[0]->name == "abs") {
          Vec e;
          if (try_const(n->kids[1], e) && e.size() == 1 && e[0] == C(2.0)) {
            Val v = gen(n->kids[0]->kids[1]);
            Val r;
            r.len = v.len;
            r.spatial = v.spatial;
            for (auto& c2 : v.c) r.c.push_back(tmp(false, "xs_abs2(" + c2 + ")"));
            return r;
          }
        }
        // conj(x).*x and x.*conj(x) -> |x|^2 (real)
        if (n->name == ".*" || n->name == "*") {
          if (is_conj_of(n->kids[0], n->kids[1]) || is_conj_of(n->kids[1], n->kids[0])) {
            const NodeP& x = is_conj_of(n->kids[0], n->kids[1]) ? n->kids[1] : n->kids[0];
            Val v = gen(x);
            Val r;
            r.len = v.len;
            r.spatial = v.spatial;
            for (auto& c : v.c) r.c.push_back(tmp(false, "xs_abs2(" + c + ")"));
            return r;
          }
        }
        return bin(n->name, gen_raw(n->kids[0]), gen_raw(n->kids[1]), n->kids[1]);
      }
      case NK::Concat: {
        Val r;
        r.len = 0;
        for (auto& row : n->rows) {
          if (row.size() != 1) throw GrammarError("horizontal concatenation is not supported; use [e1; e2]");
          Val v = gen(row[0]);
          r.cplx = r.cplx || v.cplx;
          r.spatial = r.spatial || v.spatial;
          r.len += v.len;
        }
        for (auto& row : n->rows) {
          Val v = gen(row[0]);
          for (auto& c : v.c) r.c.push_back(r.cplx && !v.cplx ? tmp(true, "mkcx(" + c + ", (real)0)") : c);
        }
        return r;
      }
      case NK::Index: return index(n);
      case NK::Colon: throw GrammarError("':' outside an index");
    }
    throw GrammarError("unsupported expression");
  }

  Val component(const Val& base, const NodeP& sel) {
    Vec k;
    if (!try_const(sel, k)) throw GrammarError("component index must be a constant");
    Val r;
    r.cplx = base.cplx;
    r.spatial = base.spatial;
    r.len = (int)k.size();
    for (auto& z : k) {
      int i = (int)z.real();
      if (i < 1 || i > base.len) throw GrammarError("component index " + std::to_string(i) + " out of range");
      r.c.push_back(base.c[i - 1]);
    }
    return r;
  }

  Val reduction(const NodeP& n, bool ave) {
    if (!ctx.allow_reduce) throw GrammarError(std::string(ave ? "Ave" : "Int") + " is only allowed in observe functions");
    if (in_integrand) throw GrammarError("nested Int/Ave is not supported");
    size_t na = n->kids.size() - 1;  // arguments
    if (na < 2) throw GrammarError("Int/Ave need the parameter struct as last argument");
    NodeP integrand = n->kids[1];
    Reduction R;
    R.ave = ave;
    std::vector<double> w(ctx.ndim + 1, 0.0);
    if (!ave) {
      for (int d = 1; d <= ctx.ndim; ++d) w[d] = ctx.dx[d];
      if (na >= 3) {
        Vec dxv;
        if (!try_const(n->kids[2], dxv)) throw GrammarError("Int step vector must be constant");
        for (int d = 1; d <= ctx.ndim; ++d) w[d] = d < (int)dxv.size() ? dxv[d].real() : 0.0;
      }
    } else {
      for (int d = 1; d <= ctx.ndim; ++d) w[d] = 1.0;
      if (na >= 3) {
        Vec av;
        if (!try_const(n->kids[2], av)) throw GrammarError("Ave switch vector must be constant");
        for (int d = 1; d <= ctx.ndim; ++d) w[d] = (d < (int)av.size() && av[d].real() > 0) ? 1.0 : 0.0;
      }
    }
    R.lo.assign(ctx.ndim + 1, 0.0);
    R.hi.assign(ctx.ndim + 1, 0.0);
    if (!ave && na >= 4) {
      auto b = n->kids[3];
      if (b->kind != NK::Concat) throw GrammarError("Int bounds must be a constant [lo hi; ...] matrix");
      for (size_t r = 0; r < b->rows.size() && (int)r <= ctx.ndim; ++r) {
        Vec row;
        for (auto& e : b->rows[r]) {
          Vec v;
          if (!try_const(e, v)) throw GrammarError("Int bounds must be constant");
          row.insert(row.end(), v.begin(), v.end());
        }
        if (row.size() != 2) throw GrammarError("Int bounds rows need two entries");
        R.lo[r] = row[0].real();
        R.hi[r] = row[1].real();
      }
    }
    if (!ave && na >= 5) throw GrammarError("Int cell argument is not supported");
    for (int d = 1; d <= ctx.ndim; ++d)
      if (w[d] > 0) { R.dims.push_back(d); R.weight.push_back(w[d]); }
    // integrand code in its own generator scope
    Gen sub(ctx);
    sub.aname = aname; sub.wname = wname; sub.vname = vname; sub.pname = pname;
    sub.kname = kname; sub.kvname = kvname; sub.xname = xname;
    sub.in_integrand = true;
    Val iv = sub.gen(integrand);
    R.lines = iv.len;
    std::ostringstream code;
    code << sub.os.str();
    for (int i = 0; i < iv.len; ++i)
      code << "  r[" << i << "] = " << (iv.cplx ? iv.c[i] : "mkcx(" + iv.c[i] + ", (real)0)") << ";\n";
    R.integrand_code = code.str();
    int base = 0;
    for (auto& q : *reds) base += q.lines;
    reds->push_back(R);
    Val r;
    r.len = iv.len;
    r.cplx = true;
    r.spatial = false;
    // Reduced over all space dims -> site independent; partial reductions stay spatial.
    if ((int)R.dims.size() < ctx.ndim) r.spatial = true;
    for (int i = 0; i < iv.len; ++i) r.c.push_back("red[" + std::to_string(base + i) + "]");
    return r;
  }

  Val index(const NodeP& n) {
    auto base = n->kids[0];
    if (base->kind == NK::Var) {
      const std::string& f = base->name;
      bool is_arg = f == aname || f == wname || f == vname || (!kname.empty() && f == kname) ||
                    (!kvname.empty() && f == kvname) || (!xname.empty() && f == xname);
      if (!is_arg) {
        if (f == "Int") return reduction(n, false);
        if (f == "Ave") return reduction(n, true);
        if (f == "xshape") {
          if (n->kids.size() < 2) throw GrammarError("xshape needs an argument");
          return gen(n->kids[1]);
        }
        if ((f == "zeros" || f == "ones") && n->kids.size() == 2 && n->kids[1]->kind == NK::Index &&
            n->kids[1]->kids[0]->kind == NK::Var && n->kids[1]->kids[0]->name == "size") {
          Val s = gen(n->kids[1]->kids[1]);
          Val r;
          r.len = s.len;
          for (int i = 0; i < s.len; ++i) r.c.push_back(f == "zeros" ? "(real)0" : "(real)1");
          return r;
        }
        if ((f == "zeros" || f == "ones") && n->kids.size() >= 2) {
          // zeros(n, 1, ...) / ones(n, 1, ...) with literal sizes: n components, broadcast over the
          // lattice and the ensemble (the other sizes must be 1)
          std::vector<int> sz;
          for (size_t i = 1; i < n->kids.size(); ++i) {
            Vec d;
            if (!try_const(n->kids[i], d) || d.size() != 1 || d[0].imag() != 0 || d[0].real() < 1 ||
                d[0].real() != std::floor(d[0].real()) || d[0].real() > 64)
              throw GrammarError(f + " takes size(x) or literal sizes (n, 1, ...)");
            sz.push_back((int)d[0].real());
          }
          for (size_t i = 1; i < sz.size(); ++i)
            if (sz[i] != 1) throw GrammarError(f + "(n, m, ...) with m > 1 is not supported on the device");
          Val r;
          r.len = sz[0];
          for (int i = 0; i < sz[0]; ++i) r.c.push_back(f == "zeros" ? "(real)0" : "(real)1");
          return r;
        }
        if (f == "sum" && (n->kids.size() == 2 || n->kids.size() == 3)) {
          Val v = gen(n->kids[1]);
          if (n->kids.size() == 3) {
            Vec d;
            if (!try_const(n->kids[2], d) || d[0].real() != 1) throw GrammarError("sum supports dimension 1 only");
          }
          Val r;
          r.cplx = v.cplx;
          r.spatial = v.spatial;
          std::string e = v.c[0];
          for (int i = 1; i < v.len; ++i) e = tmp(v.cplx, e + " + " + v.c[i]);
          r.c = {e};
          return r;
        }
        if (f == "D1" || f == "D2") {
          // D1/D2(a[, d], p) (Applications/SPDE/D1.m, D2.m): central differences of the field along
          // dimension d (2 = x), with the boundary rules of the field's boundary types
          const size_t na = n->kids.size() - 1;
          if (na != 2 && na != 3) throw GrammarError(f + " on the device takes (a, p) or (a, d, p)");
          int dd = 2;
          if (na == 3) {
            Vec dv;
            if (!try_const(n->kids[2], dv) || dv.size() != 1) throw GrammarError(f + ": the direction must be a constant");
            dd = (int)dv[0].real();
          }
          if (dd < 2 || dd - 1 > ctx.ndim) throw GrammarError(f + ": the direction must be a space dimension (2 = x)");
          const NodeP& arg = n->kids[1];
          std::vector<int> comps;
          if (arg->kind == NK::Var && arg->name == aname) {
            for (int k = 0; k < ctx.nfield; ++k) comps.push_back(k);
          } else if (arg->kind == NK::Index && arg->kids[0]->kind == NK::Var && arg->kids[0]->name == aname &&
                     arg->kids.size() >= 2) {
            Vec kv;
            if (!try_const(arg->kids[1], kv)) throw GrammarError(f + ": a(k,:) needs a constant k");
            for (auto& z : kv) {
              const int k = (int)z.real() - 1;
              if (k < 0 || k >= ctx.nfield) throw GrammarError(f + ": field component out of range");
              comps.push_back(k);
            }
          } else {
            throw GrammarError(f + " on the device takes the field a (or a(k,:)) as its first argument");
          }
          stencil = true;
          Val r;
          r.len = (int)comps.size();
          r.cplx = true;
          r.spatial = true;
          for (int k : comps)
            r.c.push_back(tmp(true, "xs_fd" + std::string(1, f[1]) + "(fld, g, s, " + std::to_string(k) + ", " +
                                        std::to_string(dd - 1) + ")"));
          return r;
        }
        if (unary_funcs().count(f)) {
          if (n->kids.size() != 2) throw GrammarError(f + " takes one argument");
          Val a = gen(n->kids[1]);
          Val r;
          r.len = a.len;
          r.spatial = a.spatial;
          bool real_out = f == "real" || f == "imag" || f == "abs" || f == "angle" || f == "floor" ||
                          f == "ceil" || f == "round" || f == "fix" || f == "erf";
          bool promote = (f == "sqrt" || f == "log" || f == "asin" || f == "acos");  // may leave the reals
          r.cplx = real_out ? false : (a.cplx || promote);
          if (f == "erf" && a.cplx) throw GrammarError("erf of a complex value is not supported");
          for (auto& c : a.c) {
            std::string arg = (promote && !a.cplx) ? "mkcx(" + c + ", (real)0)" : c;
            r.c.push_back(tmp(r.cplx, fname(f) + "(" + arg + ")"));
          }
          return r;
        }
        if ((f == "atan2" || f == "min" || f == "max" || f == "mod" || f == "rem") && n->kids.size() == 3) {
          Val a = gen(n->kids[1]), b = gen(n->kids[2]);
          if (a.cplx || b.cplx) throw GrammarError(f + " needs real arguments");
          Val r;
          r.len = std::max(a.len, b.len);
          r.spatial = a.spatial || b.spatial;
          for (int i = 0; i < r.len; ++i)
            r.c.push_back(tmp(false, fname(f) + "(" + a.c[a.len == 1 ? 0 : i] + ", " + b.c[b.len == 1 ? 0 : i] + ")"));
          return r;
        }
        throw GrammarError("unsupported function '" + f + "' (not in the device grammar)");
      }
      Val v = var(f);
      size_t na = n->kids.size() - 1;
      if (na == 0) return v;
      // a(k,:), a(k), a(:,:)
      NodeP sel = n->kids[1];
      for (size_t i = 2; i <= na; ++i)
        if (n->kids[i]->kind != NK::Colon) throw GrammarError("only the component index may be selected: use a(k,:)");
      if (sel->kind == NK::Colon) return v;
      return component(v, sel);
    }
    if (base->kind == NK::Field) {
      Vec v;
      if (try_const(n, v)) return constant(v);
      throw GrammarError("unsupported indexing of p." + base->name);
    }
    // (expr)(k,:) is not MATLAB syntax; Concat(...)(k) neither.
    throw GrammarError("unsupported indexing");
  }
};

}  // namespace

namespace {

void bind_params(Gen& g, const AnonFn& fn, const GenCtx& ctx) {
  for (size_t i = 0; i < fn.params.size() && i < ctx.roles.size(); ++i) {
    const std::string& nm = fn.params[i];
    if (nm == "~") continue;
    switch (ctx.roles[i]) {
      case Role::Field: g.aname = nm; break;
      case Role::Noise: g.wname = nm; break;
      case Role::Random: g.vname = nm; break;
      case Role::KNoise: g.kname = nm; break;
      case Role::KRandom: g.kvname = nm; break;
      case Role::Aux: g.xname = nm; break;
      case Role::Params: g.pname = nm; break;
      default: break;
    }
  }
  if (fn.params.size() > ctx.roles.size()) throw GrammarError("too many arguments in '" + fn.text + "'");
}

bool reads_var(const NodeP& n, const std::string& name) {
  if (!n) return false;
  if (n->kind == NK::Var && n->name == name) return true;
  for (auto& k : n->kids)
    if (reads_var(k, name)) return true;
  for (auto& r : n->rows)
    for (auto& e : r)
      if (reads_var(e, name)) return true;
  return false;
}

// The terms of the outermost sum of n with their signs: a - (b + c) -> +a, -b, -c.
void sum_terms(const NodeP& n, int sign, std::vector<std::pair<int, NodeP>>& out) {
  if (n->kind == NK::Bin && (n->name == "+" || n->name == "-") && n->kids.size() == 2) {
    sum_terms(n->kids[0], sign, out);
    sum_terms(n->kids[1], n->name == "-" ? -sign : sign, out);
  } else if (n->kind == NK::Un && (n->name == "-" || n->name == "+") && n->kids.size() == 1) {
    sum_terms(n->kids[0], n->name == "-" ? -sign : sign, out);
  } else {
    out.push_back({sign, n});
  }
}

}  // namespace

bool generate_split(const AnonFn& fn, const GenCtx& ctx, Generated& start, Generated& step) {
  Gen g(ctx);
  bind_params(g, fn, ctx);
  if (g.aname.empty()) return false;
  std::vector<NodeP> rows;
  if (fn.body->kind == NK::Concat) {
    for (auto& row : fn.body->rows) {
      if (row.size() != 1) return false;
      rows.push_back(row[0]);
    }
  } else {
    rows.push_back(fn.body);
  }
  std::vector<std::vector<std::pair<int, NodeP>>> rterms(rows.size());
  std::vector<int> rlen(rows.size(), 1);
  bool any_dep = false, any_inv = false;
  for (size_t r = 0; r < rows.size(); ++r) {
    sum_terms(rows[r], 1, rterms[r]);
    for (auto& [sign, t] : rterms[r]) rlen[r] = std::max(rlen[r], g.gen(t).len);
    for (auto& [sign, t] : rterms[r]) {
      if (g.gen(t).len != rlen[r] && g.gen(t).len != 1) return false;
      (reads_var(t, g.aname) ? any_dep : any_inv) = true;
    }
  }
  if (!any_dep || !any_inv) return false;
  Val hv;
  hv.c = {"h"};
  // c0 + h * (the terms that read the field, or those that do not), accumulated term by term
  auto accumulate = [&](bool dep) {
    std::vector<std::string> out;
    for (size_t r = 0; r < rows.size(); ++r) {
      Val acc;
      acc.len = rlen[r];
      acc.cplx = true;
      acc.spatial = true;
      for (int i = 0; i < rlen[r]; ++i) acc.c.push_back("c0[" + std::to_string((int)out.size() + i) + "]");
      for (auto& [sign, t] : rterms[r])
        if (reads_var(t, g.aname) == dep) acc = g.bin(sign < 0 ? "-" : "+", acc, g.gen_h(t, hv), nullptr);
      for (int i = 0; i < rlen[r]; ++i) {
        const std::string& c = acc.c[acc.len == 1 ? 0 : i];
        out.push_back(acc.cplx ? c : "mkcx(" + c + ", (real)0)");
      }
    }
    return out;
  };
  auto fill = [&](Generated& out, const std::string& body, const std::vector<std::string>& c) {
    out = Generated{};
    out.len = (int)c.size();
    out.is_complex = true;
    std::ostringstream code;
    code << body;
    for (size_t i = 0; i < c.size(); ++i) code << "  out[" << i << "] = " << c[i] << ";\n";
    out.code = code.str();
    out.stencil = g.stencil;
  };
  const std::vector<std::string> ic = accumulate(false);
  fill(start, g.os.str(), ic);
  const std::vector<std::string> sc = accumulate(true);
  fill(step, g.os.str(), sc);
  return true;
}

Generated generate(const AnonFn& fn, const GenCtx& ctx) {
  Gen g(ctx);
  std::vector<Reduction> reds;
  g.reds = &reds;
  bind_params(g, fn, ctx);
  Val v = g.gen(fn.body);
  Generated out;
  out.len = v.len;
  out.is_complex = v.cplx;
  std::ostringstream code;
  code << g.os.str();
  for (int i = 0; i < v.len; ++i)
    code << "  out[" << i << "] = " << (v.cplx ? v.c[i] : "mkcx(" + v.c[i] + ", (real)0)") << ";\n";
  out.code = code.str();
  out.reductions = reds;
  out.uses_k = false;
  out.stencil = g.stencil;
  out.spatial = v.spatial;
  return out;
}

std::vector<std::complex<double>> eval_linear(const AnonFn& fn, const GridInfo& g, const Scalars& sc,
                                              int* ncomp_out) {
  std::string pname = fn.params.empty() ? "p" : fn.params[0];
  size_t ns = 1;
  for (int d = 0; d < g.ndim; ++d) ns *= (size_t)g.n[d];
  std::vector<int> idx(g.ndim);
  std::vector<std::vector<C>> per_site;
  int ncomp = 1;
  std::vector<bool> uniform_k(g.ndim, true);
  for (int d = 0; d < g.ndim; ++d)
    for (int f = 1; f < g.nfield; ++f) uniform_k[d] = uniform_k[d] && g.k[f][d] == g.k[0][d];
  for (size_t s = 0; s < ns; ++s) {
    size_t r = s;
    for (int d = 0; d < g.ndim; ++d) {
      idx[d] = (int)(r % g.n[d]);
      r /= g.n[d];
    }
    EvalEnv env;
    env.pname = pname;
    auto kvec = [&](int d) {
      // one component when every field has the same k grid along d (all sites), else one per field
      Vec out;
      for (int f = 0; f < g.nfield; ++f) out.push_back(C(g.k[f][d][idx[d]]));
      if (uniform_k[d]) out.resize(1);
      return out;
    };
    env.field = [&](const std::string& f, Vec& out) -> bool {
      int d = -1;
      bool isD = false;
      if (f == "Dx" || f == "kx") d = 0;
      else if (f == "Dy" || f == "ky") d = 1;
      else if (f == "Dz" || f == "kz") d = 2;
      if (d >= 0) {
        if (d >= g.ndim) throw GrammarError("p." + f + " used but the problem has fewer space dimensions");
        isD = f[0] == 'D';
        out = kvec(d);
        if (isD) for (auto& z : out) z *= C(0, 1);
        return true;
      }
      if (f == "x" || f == "y" || f == "z") {
        int dd = f == "x" ? 0 : f == "y" ? 1 : 2;
        if (dd >= g.ndim) throw GrammarError("p." + f + " used but the problem has fewer space dimensions");
        out = {C(g.x[dd][idx[dd]])};
        return true;
      }
      auto it = sc.values.find(f);
      if (it != sc.values.end()) { out = {C(it->second)}; return true; }
      return false;
    };
    env.cell = [&](const std::string& f, int d, Vec& out) -> bool {
      if (f == "D" || f == "k") {
        if (d < 2 || d - 2 >= g.ndim) throw GrammarError("p." + f + "{" + std::to_string(d) + "} out of range");
        out = kvec(d - 2);
        if (f == "D") for (auto& z : out) z *= C(0, 1);
        return true;
      }
      if (f == "r") {
        if (d < 2 || d - 2 >= g.ndim) throw GrammarError("p.r{d} out of range");
        out = {C(g.x[d - 2][idx[d - 2]])};
        return true;
      }
      return false;
    };
    Vec v;
    try {
      v = eval(fn.body, env);
    } catch (const NotConst&) {
      throw GrammarError("p.linear may only use p.Dx/Dy/Dz, p.kx/ky/kz, p.D{d}, p.k{d}, coordinates and named scalars");
    }
    if (s == 0) ncomp = (int)v.size();
    if ((int)v.size() != ncomp) throw GrammarError("p.linear component count varies");
    per_site.push_back(v);
  }
  if (ncomp != 1 && ncomp != g.nfield) throw GrammarError("p.linear must have 1 or 'fields' components");
  std::vector<C> out((size_t)ncomp * ns);
  for (size_t s = 0; s < ns; ++s)
    for (int c = 0; c < ncomp; ++c) out[(size_t)c * ns + s] = per_site[s][c];
  if (ncomp_out) *ncomp_out = ncomp;
  return out;
}

}  // namespace xs
