// Initial conditions given as expressions, evaluated on the device.
//
// The reference reads each material's initial condition as an exprtk program
// from its input file and evaluates it cell by cell on the host
// (PrimeStateInitializer::GetInitialPrimeStates,
// initial_condition/prime_state_initializer.cpp:34-85, through UserExpression,
// user_expression.cpp), e.g.
//
//     if (x < 0.5) { density := 1.0; velocityX := 0.0; pressure := 1.0; }
//     else         { density := 0.125; velocityX := 0.0; pressure := 0.1; }
//
// Here the host compiles the statement subset of exprtk that ALPACA's inputs
// use into a small stack-machine program and one device thread evaluates it per
// cell. The program has forward jumps only (no loops), so every evaluation
// ends after at most its length in instructions, and its stack depth is fixed
// at compile time, so every stack index is checked before the kernel runs.
//
// Language (exprtk semantics for this subset):
//   statements   name := e;  name += e; (-=, *=, /=, %=)  var name := e;
//                if (c) S [else S]   { S ... }   e;
//                ": =" (with blanks) is read as ":=", as in the reference inputs
//   expressions  c ? a : b   if (c, a, b)   or | ||   and & &&   not !
//                < <= > >= == != <>   + -   * / %   unary - +   ^ (power,
//                not chained without parentheses)   implicit multiplication
//                after a number or ')' ("2(x + 1)", "2x")
//   functions    abs acos acosh asin asinh atan atanh cbrt ceil cos cosh exp
//                expm1 floor frac log log10 log1p log2 round sgn sin sinh sqrt
//                tan tanh trunc deg2rad rad2deg; atan2 hypot pow logn root;
//                min max (two or more arguments)
//   symbols      x y z (cell centre), pi, true false, the prime states
//                density velocityX velocityY velocityZ pressure (initially 0)
//   comments     // ... , # ... , /* ... */
// Truth values are doubles (0 false); "and"/"or" evaluate both sides;
// a == b when |a - b| <= 1e-10 max(1, |a|, |b|) (exprtk's floating-point
// equality).
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/alpaca_b200.h"
#include "kernels.cuh"
#include "layout.cuh"
#include "numerics.cuh"
#include "engine.hpp"

namespace alp {
int fail(int code, const std::string &msg);
}

namespace alp {
namespace expr {

enum Op : int {
  OP_CONST, OP_LOAD, OP_STORE, OP_POP,
  OP_ADD, OP_SUB, OP_MUL, OP_DIV, OP_MOD, OP_POW, OP_NEG,
  OP_LT, OP_LE, OP_GT, OP_GE, OP_EQ, OP_NE, OP_AND, OP_OR, OP_NOT,
  OP_F1, OP_F2, OP_MIN, OP_MAX, OP_JZ, OP_JMP, OP_END
};
static const char *const kOpNames[] = {
    "CONST", "LOAD", "STORE", "POP", "ADD", "SUB", "MUL", "DIV", "MOD", "POW", "NEG",
    "LT", "LE", "GT", "GE", "EQ", "NE", "AND", "OR", "NOT", "F1", "F2", "MIN", "MAX",
    "JZ", "JMP", "END"};

static const char *const kF1[] = {"abs", "acos", "acosh", "asin", "asinh", "atan", "atanh",
                                  "cbrt", "ceil", "cos", "cosh", "exp", "expm1", "floor",
                                  "frac", "log", "log10", "log1p", "log2", "round", "sgn",
                                  "sin", "sinh", "sqrt", "tan", "tanh", "trunc", "deg2rad",
                                  "rad2deg"};
static const char *const kF2[] = {"atan2", "hypot", "pow", "logn", "root"};
constexpr int NF1 = sizeof(kF1) / sizeof(kF1[0]);
constexpr int NF2 = sizeof(kF2) / sizeof(kF2[0]);

// variable slots: the cell centre, the prime states, then local variables
static const char *const kSlots[] = {"x", "y", "z", "density", "velocityX", "velocityY",
                                     "velocityZ", "pressure"};
constexpr int SLOT_PRIME = 3;
constexpr int MAX_SLOTS = 32, MAX_STACK = 32, MAX_CODE = 1 << 16;

struct Ins {
  int op, arg;
};

struct Program {
  std::vector<Ins> code;
  std::vector<double> consts;
  std::vector<std::string> names;  // slot names
  int max_stack = 0;
  // device copy, made on first use
  Ins *d_code = nullptr;
  double *d_consts = nullptr;
};

// ---- lexer -----------------------------------------------------------------

enum Tok { T_END, T_NUM, T_ID, T_OP };
struct Token {
  Tok kind;
  std::string text;
  double value;
  size_t pos;
};

struct ParseError {
  std::string msg;
  size_t pos;
};

static std::vector<Token> lex(const std::string &s) {
  std::vector<Token> out;
  size_t i = 0, n = s.size();
  while (true) {
    while (i < n) {
      if (isspace((unsigned char)s[i])) {
        ++i;
      } else if (s[i] == '#' || (s[i] == '/' && i + 1 < n && s[i + 1] == '/')) {
        while (i < n && s[i] != '\n') ++i;
      } else if (s[i] == '/' && i + 1 < n && s[i + 1] == '*') {
        size_t const e = s.find("*/", i + 2);
        if (e == std::string::npos) throw ParseError{"unterminated comment", i};
        i = e + 2;
      } else {
        break;
      }
    }
    if (i >= n) {
      out.push_back({T_END, "", 0.0, i});
      return out;
    }
    size_t const p = i;
    char const c = s[i];
    if (isdigit((unsigned char)c) || (c == '.' && i + 1 < n && isdigit((unsigned char)s[i + 1]))) {
      char *end = nullptr;
      double const v = strtod(s.c_str() + i, &end);
      size_t const len = (size_t)(end - (s.c_str() + i));
      out.push_back({T_NUM, s.substr(i, len), v, p});
      i += len;
    } else if (isalpha((unsigned char)c) || c == '_') {
      size_t j = i;
      while (j < n && (isalnum((unsigned char)s[j]) || s[j] == '_')) ++j;
      out.push_back({T_ID, s.substr(i, j - i), 0.0, p});
      i = j;
    } else if (c == ':') {
      size_t j = i + 1;
      while (j < n && (s[j] == ' ' || s[j] == '\t')) ++j;
      if (j < n && s[j] == '=' && !(j + 1 < n && s[j + 1] == '=')) {
        out.push_back({T_OP, ":=", 0.0, p});
        i = j + 1;
      } else {
        out.push_back({T_OP, ":", 0.0, p});
        ++i;
      }
    } else {
      static const char *const two[] = {"+=", "-=", "*=", "/=", "%=", "<=", ">=", "==", "!=",
                                        "<>", "&&", "||"};
      std::string op(1, c);
      for (auto t : two)
        if (s.compare(i, 2, t) == 0) op = t;
      if (op.size() == 1 && !strchr("+-*/%^<>=!&|(){},;?[]", c))
        throw ParseError{std::string("unexpected character '") + c + "'", p};
      out.push_back({T_OP, op, 0.0, p});
      i += op.size();
    }
  }
}

// ---- parser and code generator ---------------------------------------------

class Compiler {
 public:
  explicit Compiler(std::vector<Token> t) : tok_(std::move(t)) {
    for (auto s : kSlots) prog_.names.push_back(s);
  }

  Program run() {
    while (!at_end()) statement();
    emit(OP_END, 0);
    if (depth_ != 0) throw ParseError{"internal: unbalanced stack", 0};
    prog_.max_stack = max_depth_;
    return std::move(prog_);
  }

 private:
  std::vector<Token> tok_;
  size_t k_ = 0;
  Program prog_;
  int depth_ = 0, max_depth_ = 0;

  Token const &cur() const { return tok_[k_]; }
  bool at_end() const { return cur().kind == T_END; }
  bool is_op(const char *o) const { return cur().kind == T_OP && cur().text == o; }
  bool is_id(const char *o) const { return cur().kind == T_ID && cur().text == o; }
  [[noreturn]] void error(const std::string &m) const { throw ParseError{m, cur().pos}; }
  void expect(const char *o) {
    if (!is_op(o)) error(std::string("expected '") + o + "'" + found());
    ++k_;
  }
  std::string found() const {
    return at_end() ? " at the end of the expression" : " before '" + cur().text + "'";
  }

  int emit(int op, int arg) {
    if (prog_.code.size() >= (size_t)MAX_CODE) error("program too long");
    prog_.code.push_back({op, arg});
    switch (op) {
      case OP_CONST: case OP_LOAD: push(1); break;
      case OP_STORE: case OP_POP: case OP_JZ: push(-1); break;
      case OP_ADD: case OP_SUB: case OP_MUL: case OP_DIV: case OP_MOD: case OP_POW:
      case OP_LT: case OP_LE: case OP_GT: case OP_GE: case OP_EQ: case OP_NE:
      case OP_AND: case OP_OR: case OP_F2: case OP_MIN: case OP_MAX: push(-1); break;
      default: break;
    }
    return (int)prog_.code.size() - 1;
  }
  void push(int d) {
    depth_ += d;
    if (depth_ > max_depth_) max_depth_ = depth_;
    if (max_depth_ > MAX_STACK) error("expression nested too deeply");
  }
  void patch(int at) { prog_.code[at].arg = (int)prog_.code.size(); }
  int constant(double v) {
    prog_.consts.push_back(v);
    return (int)prog_.consts.size() - 1;
  }
  int slot(const std::string &name) const {
    for (size_t s = 0; s < prog_.names.size(); ++s)
      if (prog_.names[s] == name) return (int)s;
    return -1;
  }

  static bool keyword(const std::string &w) {
    return w == "if" || w == "else" || w == "var" || w == "and" || w == "or" || w == "not" ||
           w == "true" || w == "false";
  }

  // -- statements --
  void statement() {
    if (is_op(";")) {
      ++k_;
      return;
    }
    if (is_op("{")) {
      ++k_;
      while (!is_op("}")) {
        if (at_end()) error("expected '}'");
        statement();
      }
      ++k_;
      return;
    }
    if (is_id("if") && k_ + 1 < tok_.size() && tok_[k_ + 1].text == "(" && !if_is_function()) {
      if_statement();
      return;
    }
    if (is_id("var")) {
      ++k_;
      if (cur().kind != T_ID || keyword(cur().text)) error("expected a variable name");
      std::string const name = cur().text;
      if (slot(name) >= 0) error("'" + name + "' is already defined");
      if (prog_.names.size() >= (size_t)MAX_SLOTS) error("too many variables");
      prog_.names.push_back(name);
      int const s = (int)prog_.names.size() - 1;
      ++k_;
      if (is_op(":=")) {
        ++k_;
        expression();
      } else {
        emit(OP_CONST, constant(0.0));
      }
      emit(OP_STORE, s);
      end_statement();
      return;
    }
    if (cur().kind == T_ID && k_ + 1 < tok_.size() && tok_[k_ + 1].kind == T_OP) {
      std::string const a = tok_[k_ + 1].text;
      if (a == ":=" || a == "+=" || a == "-=" || a == "*=" || a == "/=" || a == "%=") {
        std::string const name = cur().text;
        int const s = slot(name);
        if (s < 0) error("assignment to unknown variable '" + name + "'");
        if (s < SLOT_PRIME) error("the cell centre '" + name + "' cannot be assigned");
        k_ += 2;
        if (a != ":=") emit(OP_LOAD, s);
        expression();
        if (a == "+=") emit(OP_ADD, 0);
        if (a == "-=") emit(OP_SUB, 0);
        if (a == "*=") emit(OP_MUL, 0);
        if (a == "/=") emit(OP_DIV, 0);
        if (a == "%=") emit(OP_MOD, 0);
        emit(OP_STORE, s);
        end_statement();
        return;
      }
    }
    expression();
    emit(OP_POP, 0);
    end_statement();
  }
  void end_statement() {
    if (is_op(";")) {
      ++k_;
    } else if (!at_end() && !is_op("}")) {
      error("expected ';'" + found());
    }
  }
  // "if (c, a, b)" is an expression; "if (c) S" a statement
  bool if_is_function() const {
    int level = 0;
    for (size_t j = k_ + 1; j < tok_.size(); ++j) {
      auto const &t = tok_[j];
      if (t.kind == T_END) return false;
      if (t.kind != T_OP) continue;
      if (t.text == "(" || t.text == "{" || t.text == "[") ++level;
      if (t.text == ")" || t.text == "}" || t.text == "]") {
        if (--level == 0) return false;
      }
      if (t.text == "," && level == 1) return true;
    }
    return false;
  }
  void if_statement() {
    ++k_;
    expect("(");
    expression();
    expect(")");
    int const jz = emit(OP_JZ, 0);
    branch_body();
    if (is_id("else")) {
      ++k_;
      int const jmp = emit(OP_JMP, 0);
      patch(jz);
      branch_body();
      patch(jmp);
    } else {
      patch(jz);
    }
  }
  void branch_body() {
    if (at_end()) error("expected a statement");
    statement();
  }

  // -- expressions (each leaves one value on the stack) --
  void expression() { ternary(); }
  void ternary() {
    logical_or();
    if (is_op("?")) {
      ++k_;
      int const jz = emit(OP_JZ, 0);
      int const d = depth_;
      ternary();
      int const jmp = emit(OP_JMP, 0);
      patch(jz);
      depth_ = d;
      expect(":");
      ternary();
      patch(jmp);
    }
  }
  void logical_or() {
    logical_and();
    while (is_op("|") || is_op("||") || is_id("or")) {
      ++k_;
      logical_and();
      emit(OP_OR, 0);
    }
  }
  void logical_and() {
    comparison();
    while (is_op("&") || is_op("&&") || is_id("and")) {
      ++k_;
      comparison();
      emit(OP_AND, 0);
    }
  }
  void comparison() {
    additive();
    while (true) {
      int op = -1;
      if (is_op("<")) op = OP_LT;
      else if (is_op("<=")) op = OP_LE;
      else if (is_op(">")) op = OP_GT;
      else if (is_op(">=")) op = OP_GE;
      else if (is_op("==") || is_op("=")) op = OP_EQ;
      else if (is_op("!=") || is_op("<>")) op = OP_NE;
      if (op < 0) return;
      ++k_;
      additive();
      emit(op, 0);
    }
  }
  void additive() {
    multiplicative();
    while (is_op("+") || is_op("-")) {
      int const op = is_op("+") ? OP_ADD : OP_SUB;
      ++k_;
      multiplicative();
      emit(op, 0);
    }
  }
  bool starts_implicit_factor() const {
    if (is_op("(")) return true;
    return cur().kind == T_ID && !keyword(cur().text);
  }
  void multiplicative() {
    bool implicit_ok = unary();
    while (true) {
      if (is_op("*") || is_op("/") || is_op("%")) {
        int const op = is_op("*") ? OP_MUL : (is_op("/") ? OP_DIV : OP_MOD);
        ++k_;
        implicit_ok = unary();
        emit(op, 0);
      } else if (implicit_ok && starts_implicit_factor()) {
        implicit_ok = unary();
        emit(OP_MUL, 0);
      } else {
        return;
      }
    }
  }
  // returns whether the factor may be followed by an implicit multiplication
  // (it ended with a number or a closing parenthesis)
  bool unary() {
    if (is_op("-")) {
      ++k_;
      bool const ok = unary();
      emit(OP_NEG, 0);
      return ok;
    }
    if (is_op("+")) {
      ++k_;
      return unary();
    }
    if (is_op("!") || is_id("not")) {
      ++k_;
      unary();
      emit(OP_NOT, 0);
      return false;
    }
    bool const ok = primary();
    if (is_op("^")) {
      ++k_;
      if (is_op("-")) {
        ++k_;
        primary();
        emit(OP_NEG, 0);
      } else {
        if (is_op("+")) ++k_;
        primary();
      }
      emit(OP_POW, 0);
      if (is_op("^")) error("chained '^': use parentheses");
      return false;
    }
    return ok;
  }
  int arguments() {
    expect("(");
    int n = 0;
    if (!is_op(")")) {
      while (true) {
        expression();
        ++n;
        if (is_op(",")) {
          ++k_;
          continue;
        }
        break;
      }
    }
    expect(")");
    return n;
  }
  bool primary() {
    Token const t = cur();
    if (t.kind == T_NUM) {
      ++k_;
      emit(OP_CONST, constant(t.value));
      return true;
    }
    if (is_op("(")) {
      ++k_;
      expression();
      expect(")");
      return true;
    }
    if (t.kind != T_ID) error("expected a value" + found());
    std::string const w = t.text;
    ++k_;
    if (w == "if") {
      expect("(");
      expression();
      expect(",");
      int const jz = emit(OP_JZ, 0);
      int const d = depth_;
      expression();
      int const jmp = emit(OP_JMP, 0);
      patch(jz);
      depth_ = d;
      expect(",");
      expression();
      expect(")");
      patch(jmp);
      return true;
    }
    if (w == "pi") {
      emit(OP_CONST, constant(3.14159265358979323846));
      return false;
    }
    if (w == "true" || w == "false") {
      emit(OP_CONST, constant(w == "true" ? 1.0 : 0.0));
      return false;
    }
    for (int f = 0; f < NF1; ++f)
      if (w == kF1[f]) {
        if (arguments() != 1) error("'" + w + "' takes one argument");
        emit(OP_F1, f);
        return true;
      }
    for (int f = 0; f < NF2; ++f)
      if (w == kF2[f]) {
        if (arguments() != 2) error("'" + w + "' takes two arguments");
        emit(OP_F2, f);
        return true;
      }
    if (w == "min" || w == "max") {
      int const n = arguments();
      if (n < 2) error("'" + w + "' takes at least two arguments");
      for (int a = 1; a < n; ++a) emit(w == "min" ? OP_MIN : OP_MAX, 0);
      return true;
    }
    int const s = slot(w);
    if (s < 0 || keyword(w)) {
      --k_;
      error("unknown symbol '" + w + "'");
    }
    emit(OP_LOAD, s);
    return false;
  }
};

// ---- evaluation ------------------------------------------------------------

__host__ __device__ inline double f1(int f, double a) {
  switch (f) {
    case 0: return fabs(a);
    case 1: return acos(a);
    case 2: return acosh(a);
    case 3: return asin(a);
    case 4: return asinh(a);
    case 5: return atan(a);
    case 6: return atanh(a);
    case 7: return cbrt(a);
    case 8: return ceil(a);
    case 9: return cos(a);
    case 10: return cosh(a);
    case 11: return exp(a);
    case 12: return expm1(a);
    case 13: return floor(a);
    case 14: return a - trunc(a);
    case 15: return log(a);
    case 16: return log10(a);
    case 17: return log1p(a);
    case 18: return log2(a);
    case 19: return round(a);
    case 20: return a > 0.0 ? 1.0 : (a < 0.0 ? -1.0 : 0.0);
    case 21: return sin(a);
    case 22: return sinh(a);
    case 23: return sqrt(a);
    case 24: return tan(a);
    case 25: return tanh(a);
    case 26: return trunc(a);
    case 27: return a * (3.14159265358979323846 / 180.0);
    default: return a * (180.0 / 3.14159265358979323846);
  }
}
__host__ __device__ inline double f2(int f, double a, double b) {
  switch (f) {
    case 0: return atan2(a, b);
    case 1: return hypot(a, b);
    case 2: return pow(a, b);
    case 3: return log(a) / log(b);
    default: return pow(a, 1.0 / b);
  }
}
__host__ __device__ inline double truth(bool b) { return b ? 1.0 : 0.0; }
__host__ __device__ inline bool feq(double a, double b) {
  double const m = fmax(1.0, fmax(fabs(a), fabs(b)));
  return fabs(a - b) <= 1e-10 * m;
}

// What one launch evaluates: the program, where the nodes are (an explicit
// origin per node, or a regular grid of nodes from a domain origin), the unit
// references and the output (prime states, or conservatives in engine blocks).
struct ExprLaunch {
  Ins const *code;
  double const *consts;
  double const *origins;  // [nb][3], or null for the regular grid below
  double o[3];            // domain origin of the regular grid
  int nby, nbz;           // nodes along y and z of the regular grid
  double h;               // dimensional cell size
  double rho_ref, vel_ref, p_ref;
  double *prims;  // [nb][DIM+2][IC^d] non-dimensional rho, p, u.. (the reference's order)
  double *U;      // or the engine's block pool, blocks first.. first+nb-1
  int first;
  double gamma, B;
};

// One thread per interior cell of node blockIdx.y. The program's stack depth
// was checked against MAX_STACK when it was compiled, and its jumps only go
// forward, so the loop ends at OP_END after at most the program's length.
template <int DIM>
__global__ void expr_ic_kernel(ExprLaunch L) {
  using G = Geo<DIM>;
  constexpr int CELLS = G::ICX * G::ICY * G::ICZ;
  int const c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= CELLS) return;
  int const b = blockIdx.y;
  int const k = c % G::ICZ, j = (c / G::ICZ) % G::ICY, i = c / (G::ICZ * G::ICY);
  double org[3];
  if (L.origins) {
    for (int d = 0; d < 3; ++d) org[d] = L.origins[3 * b + d];
  } else {
    int const bx = b / (L.nby * L.nbz), by = (b / L.nbz) % L.nby, bz = b % L.nbz;
    org[0] = L.o[0] + bx * (IC * L.h);
    org[1] = L.o[1] + by * (IC * L.h);
    org[2] = L.o[2] + bz * (IC * L.h);
  }
  double var[MAX_SLOTS];
  double st[MAX_STACK];
  for (int s = 0; s < MAX_SLOTS; ++s) var[s] = 0.0;
  var[0] = org[0] + (i + 0.5) * L.h;
  var[1] = DIM > 1 ? org[1] + (j + 0.5) * L.h : 0.0;
  var[2] = DIM > 2 ? org[2] + (k + 0.5) * L.h : 0.0;
  int sp = 0;
  for (int pc = 0; pc < MAX_CODE; ++pc) {
    Ins const in = L.code[pc];
    switch (in.op) {
      case OP_CONST: st[sp++] = L.consts[in.arg]; continue;
      case OP_LOAD: st[sp++] = var[in.arg]; continue;
      case OP_STORE: var[in.arg] = st[--sp]; continue;
      case OP_POP: --sp; continue;
      case OP_NEG: st[sp - 1] = -st[sp - 1]; continue;
      case OP_NOT: st[sp - 1] = truth(st[sp - 1] == 0.0); continue;
      case OP_F1: st[sp - 1] = f1(in.arg, st[sp - 1]); continue;
      case OP_JZ:
        if (st[--sp] == 0.0) pc = in.arg - 1;
        continue;
      case OP_JMP: pc = in.arg - 1; continue;
      case OP_END: pc = MAX_CODE; continue;
      default: break;
    }
    double const a = st[sp - 2], bb = st[sp - 1];
    double r;
    switch (in.op) {
      case OP_ADD: r = a + bb; break;
      case OP_SUB: r = a - bb; break;
      case OP_MUL: r = a * bb; break;
      case OP_DIV: r = a / bb; break;
      case OP_MOD: r = fmod(a, bb); break;
      case OP_POW: r = pow(a, bb); break;
      case OP_LT: r = truth(a < bb); break;
      case OP_LE: r = truth(a <= bb); break;
      case OP_GT: r = truth(a > bb); break;
      case OP_GE: r = truth(a >= bb); break;
      case OP_EQ: r = truth(feq(a, bb)); break;
      case OP_NE: r = truth(!feq(a, bb)); break;
      case OP_AND: r = truth(a != 0.0 && bb != 0.0); break;
      case OP_OR: r = truth(a != 0.0 || bb != 0.0); break;
      case OP_F2: r = f2(in.arg, a, bb); break;
      case OP_MIN: r = fmin(a, bb); break;
      default: r = fmax(a, bb); break;  // OP_MAX
    }
    st[sp - 2] = r;
    --sp;
  }
  // non-dimensional prime states (unit_handler.cpp:67-98)
  double const rho = var[SLOT_PRIME + 0] / L.rho_ref;
  double vel[3] = {0.0, 0.0, 0.0};
  for (int d = 0; d < DIM; ++d) vel[d] = var[SLOT_PRIME + 1 + d] / L.vel_ref;
  double const p = var[SLOT_PRIME + 4] / L.p_ref;
  if (L.prims) {
    // PrimeState order Density, Pressure, VelocityX.. (block_definitions/field_details.h:201-212)
    double *out = L.prims + (size_t)b * (DIM + 2) * CELLS;
    out[c] = rho;
    out[CELLS + c] = p;
    for (int d = 0; d < DIM; ++d) out[(2 + d) * CELLS + c] = vel[d];
  } else {
    // PrimeStatesToConservatives (prime_states/prime_state_handler.h:195-275)
    Eos const eos{L.gamma, L.B, 0};
    double *ub = L.U + (size_t)(L.first + b) * G::BLOCK_DOUBLES;
    int const x = ((i + HS) * G::TCY + (j + (DIM > 1 ? HS : 0))) * G::TCZ + (k + (DIM > 2 ? HS : 0));
    ub[MASS * G::CELLS + x] = rho;
    for (int d = 0; d < DIM; ++d) ub[(MOMX + d) * G::CELLS + x] = vel[d] * rho;
    ub[ENERGY * G::CELLS + x] = eos_energy<DIM, double>(eos, rho, vel[0], vel[1], vel[2], p);
  }
}

}  // namespace expr
}  // namespace alp

using namespace alp;
using namespace alp::expr;

struct alp_ic_program {
  Program p;
};

namespace {

int upload(alp_ic_program *prog) {
  Program &p = prog->p;
  if (p.d_code) return ALP_OK;
  if (cudaMalloc(&p.d_code, p.code.size() * sizeof(Ins)) != cudaSuccess ||
      cudaMalloc(&p.d_consts, (p.consts.size() + 1) * sizeof(double)) != cudaSuccess) {
    cudaFree(p.d_code);
    p.d_code = nullptr;
    return fail(ALP_ERR_CUDA, "cannot allocate the program on the device");
  }
  if (cudaMemcpy(p.d_code, p.code.data(), p.code.size() * sizeof(Ins), cudaMemcpyHostToDevice) !=
          cudaSuccess ||
      (!p.consts.empty() && cudaMemcpy(p.d_consts, p.consts.data(),
                                       p.consts.size() * sizeof(double),
                                       cudaMemcpyHostToDevice) != cudaSuccess))
    return fail(ALP_ERR_CUDA, "cannot copy the program to the device");
  return ALP_OK;
}

// program on the device, unit references and dimensional cell size
int prepare(const alp_ic_program *prog, const alp_units *u, double cell_size, ExprLaunch &L) {
  double const rho = u ? u->density : 1.0, vel = u ? u->velocity : 1.0, len = u ? u->length : 1.0;
  if (!(rho > 0.0) || !(vel > 0.0) || !(len > 0.0))
    return fail(ALP_ERR_INVALID, "reference density, velocity and length must be positive");
  if (int rc = upload(const_cast<alp_ic_program *>(prog))) return rc;
  L.code = prog->p.d_code;
  L.consts = prog->p.d_consts;
  L.h = cell_size * len;
  L.rho_ref = rho;
  L.vel_ref = vel;
  L.p_ref = rho * vel * vel;  // unit_handler.cpp:45-46
  L.nby = L.nbz = 1;
  return ALP_OK;
}

int launch(int dim, int nb, ExprLaunch const &L, cudaStream_t s) {
  int const cells = dim == 1 ? IC : (dim == 2 ? IC * IC : IC * IC * IC);
  dim3 const grid((cells + 127) / 128, nb);
  switch (dim) {
    case 1: expr_ic_kernel<1><<<grid, 128, 0, s>>>(L); break;
    case 2: expr_ic_kernel<2><<<grid, 128, 0, s>>>(L); break;
    default: expr_ic_kernel<3><<<grid, 128, 0, s>>>(L); break;
  }
  cudaError_t const e = cudaGetLastError();
  if (e != cudaSuccess) return fail(ALP_ERR_CUDA, std::string("initial condition: ") + cudaGetErrorString(e));
  return ALP_OK;
}

}  // namespace

extern "C" {

int alp_ic_program_create(const char *text, alp_ic_program **out) {
  if (!text || !out) return fail(ALP_ERR_INVALID, "null argument");
  *out = nullptr;
  try {
    Compiler c(lex(text));
    auto *p = new alp_ic_program{c.run()};
    *out = p;
    return ALP_OK;
  } catch (ParseError const &e) {
    return fail(ALP_ERR_INVALID, "initial-condition expression, position " +
                                     std::to_string(e.pos) + ": " + e.msg);
  } catch (std::exception const &e) {
    return fail(ALP_ERR_INVALID, std::string("initial-condition expression: ") + e.what());
  }
}

void alp_ic_program_destroy(alp_ic_program *p) {
  if (!p) return;
  cudaFree(p->p.d_code);
  cudaFree(p->p.d_consts);
  delete p;
}

int alp_ic_program_listing(const alp_ic_program *prog, char *buf, int size, int *written) {
  if (!prog || !buf || size <= 0) return fail(ALP_ERR_INVALID, "null argument");
  std::string s;
  char line[96];
  for (auto const &in : prog->p.code) {
    std::string arg;
    if (in.op == OP_CONST) {
      snprintf(line, sizeof line, "%.17g", prog->p.consts[in.arg]);
      arg = line;
    } else if (in.op == OP_LOAD || in.op == OP_STORE) {
      arg = prog->p.names[in.arg];
    } else if (in.op == OP_F1) {
      arg = kF1[in.arg];
    } else if (in.op == OP_F2) {
      arg = kF2[in.arg];
    } else if (in.op == OP_JZ || in.op == OP_JMP) {
      arg = std::to_string(in.arg);
    }
    s += kOpNames[in.op];
    if (!arg.empty()) s += " " + arg;
    s += "\n";
  }
  if (written) *written = (int)s.size();
  if ((int)s.size() >= size) return fail(ALP_ERR_INVALID, "listing buffer too small");
  memcpy(buf, s.c_str(), s.size() + 1);
  return ALP_OK;
}

int alp_ic_program_info(const alp_ic_program *prog, int *n_instructions, int *max_stack,
                        int *n_variables) {
  if (!prog) return fail(ALP_ERR_INVALID, "null program");
  if (n_instructions) *n_instructions = (int)prog->p.code.size();
  if (max_stack) *max_stack = prog->p.max_stack;
  if (n_variables) *n_variables = (int)prog->p.names.size();
  return ALP_OK;
}

int alp_ic_evaluate(const alp_ic_program *prog, int dim, int nb, const double *d_origins,
                    double cell_size, const alp_units *units, double *d_prims, void *stream) {
  if (!prog || !d_origins || !d_prims) return fail(ALP_ERR_INVALID, "null argument");
  if (dim < 1 || dim > 3) return fail(ALP_ERR_INVALID, "dimension must be 1, 2 or 3");
  if (nb < 0 || nb > 65535) return fail(ALP_ERR_INVALID, "between 0 and 65535 nodes per call");
  if (nb == 0) return ALP_OK;
  if (!(cell_size > 0.0)) return fail(ALP_ERR_INVALID, "cell size must be positive");
  ExprLaunch L{};
  if (int rc = prepare(prog, units, cell_size, L)) return rc;
  L.origins = d_origins;
  L.prims = d_prims;
  return launch(dim, nb, L, (cudaStream_t)stream);
}

int alp_engine_add_case_expr(alp_engine *e, const alp_material *mat, double cell_size,
                             double cfl, double t0, double t_end, int max_steps,
                             const int *nblocks, const int *periodic, const double *origin,
                             const alp_units *units, const alp_ic_program *prog, int *case_id) {
  if (!e || !case_id || !nblocks || !periodic || !prog || !mat)
    return fail(ALP_ERR_INVALID, "null argument");
  int n[3] = {1, 1, 1};
  for (int d = 0; d < e->dim; ++d) {
    if (nblocks[d] <= 0) return fail(ALP_ERR_INVALID, "block counts must be positive");
    n[d] = nblocks[d];
  }
  int const nb = n[0] * n[1] * n[2];
  if (nb > 65535) return fail(ALP_ERR_INVALID, "at most 65535 blocks per case");
  if (!(cell_size > 0.0)) return fail(ALP_ERR_INVALID, "cell size must be positive");
  ExprLaunch L{};
  if (int rc = prepare(prog, units, cell_size, L)) return rc;
  std::vector<int> nbr = regular_grid_neighbours(e->dim, n, periodic);
  int cid, first;
  if (int rc = engine_add_case_core(e, mat, cell_size, cfl, t0, t_end, max_steps, nb, nbr.data(),
                                    &cid, &first))
    return rc;
  for (int d = 0; d < 3; ++d) L.o[d] = (origin && d < e->dim) ? origin[d] : 0.0;
  L.nby = n[1];
  L.nbz = n[2];
  L.U = e->U;
  L.first = first;
  L.gamma = mat->gamma;
  L.B = mat->background_pressure;
  if (int rc = launch(e->dim, nb, L, e->stream)) {
    alp_engine_remove_case(e, cid);
    return rc;
  }
  *case_id = cid;
  return ALP_OK;
}

}  // extern "C"
