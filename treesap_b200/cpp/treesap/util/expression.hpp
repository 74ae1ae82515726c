// treesap-b200: run-time math expressions of x, y, z compiled on the host into a flat postfix
// program that the host and the device evaluate with a small stack machine. Stands in for
// the amrex::Parser that the reference's FunctionInit uses (init/FunctionInit.hpp:34-101).
//
// Grammar (the operators and functions of AMReX's parser that initial conditions use):
//   expr    := or
//   or      := and  (("||" | "or")  and)*
//   and     := cmp  (("&&" | "and") cmp)*
//   cmp     := add  (("<" | ">" | "<=" | ">=" | "==" | "!=") add)?
//   add     := mul  (("+" | "-") mul)*
//   mul     := unary (("*" | "/") unary)*
//   unary   := ("-" | "+") unary | power
//   power   := primary (("^" | "**") unary)?          right-associative: 2^3^2 = 2^9, -x^2 = -(x^2)
//   primary := number | x | y | z | pi | name "(" expr ("," expr)* ")" | "(" expr ")"
// Functions: sin cos tan asin acos atan sinh cosh tanh exp log log10 sqrt abs fabs floor ceil
// erf heaviside (1 argument); pow atan2 min max fmod (2); if(cond, a, b) (3, both branches
// are evaluated). Comparisons and logical operators give 1 or 0.
#pragma once

#include <AMReX.H>

#include <cctype>
#include <cmath>
#include <stdexcept>
#include <string>
#include <vector>

namespace treesap {
namespace expr {

enum Op : int {
    kConst,
    kX,
    kY,
    kZ,
    kAdd,
    kSub,
    kMul,
    kDiv,
    kPow,
    kNeg,
    kLt,
    kGt,
    kLe,
    kGe,
    kEq,
    kNe,
    kAnd,
    kOr,
    kSin,
    kCos,
    kTan,
    kAsin,
    kAcos,
    kAtan,
    kSinh,
    kCosh,
    kTanh,
    kExp,
    kLog,
    kLog10,
    kSqrt,
    kAbs,
    kFloor,
    kCeil,
    kErf,
    kHeaviside,
    kAtan2,
    kMin,
    kMax,
    kFmod,
    kIf
};

/// One postfix instruction (kConst carries its value).
struct Instr {
    int op;
    double value;
};

constexpr int kMaxStack = 32;

/// Evaluates a postfix program at (x, y, z).
AMREX_GPU_HOST_DEVICE inline double eval(const Instr* code, int n, double x, double y, double z) {
    double st[kMaxStack];
    int sp = 0;
    for (int q = 0; q < n; ++q) {
        const Instr in = code[q];
        switch (in.op) {
        case kConst: st[sp++] = in.value; break;
        case kX: st[sp++] = x; break;
        case kY: st[sp++] = y; break;
        case kZ: st[sp++] = z; break;
        case kNeg: st[sp - 1] = -st[sp - 1]; break;
        case kSin: st[sp - 1] = sin(st[sp - 1]); break;
        case kCos: st[sp - 1] = cos(st[sp - 1]); break;
        case kTan: st[sp - 1] = tan(st[sp - 1]); break;
        case kAsin: st[sp - 1] = asin(st[sp - 1]); break;
        case kAcos: st[sp - 1] = acos(st[sp - 1]); break;
        case kAtan: st[sp - 1] = atan(st[sp - 1]); break;
        case kSinh: st[sp - 1] = sinh(st[sp - 1]); break;
        case kCosh: st[sp - 1] = cosh(st[sp - 1]); break;
        case kTanh: st[sp - 1] = tanh(st[sp - 1]); break;
        case kExp: st[sp - 1] = exp(st[sp - 1]); break;
        case kLog: st[sp - 1] = log(st[sp - 1]); break;
        case kLog10: st[sp - 1] = log10(st[sp - 1]); break;
        case kSqrt: st[sp - 1] = sqrt(st[sp - 1]); break;
        case kAbs: st[sp - 1] = fabs(st[sp - 1]); break;
        case kFloor: st[sp - 1] = floor(st[sp - 1]); break;
        case kCeil: st[sp - 1] = ceil(st[sp - 1]); break;
        case kErf: st[sp - 1] = erf(st[sp - 1]); break;
        case kHeaviside: st[sp - 1] = st[sp - 1] > 0.0 ? 1.0 : 0.0; break;
        case kIf: {
            const double c = st[sp - 3], a = st[sp - 2], b = st[sp - 1];
            sp -= 2;
            st[sp - 1] = c != 0.0 ? a : b;
            break;
        }
        default: {
            const double b = st[--sp], a = st[sp - 1];
            double r = 0.0;
            switch (in.op) {
            case kAdd: r = a + b; break;
            case kSub: r = a - b; break;
            case kMul: r = a * b; break;
            case kDiv: r = a / b; break;
            case kPow: r = pow(a, b); break;
            case kLt: r = a < b; break;
            case kGt: r = a > b; break;
            case kLe: r = a <= b; break;
            case kGe: r = a >= b; break;
            case kEq: r = a == b; break;
            case kNe: r = a != b; break;
            case kAnd: r = (a != 0.0) && (b != 0.0); break;
            case kOr: r = (a != 0.0) || (b != 0.0); break;
            case kAtan2: r = atan2(a, b); break;
            case kMin: r = fmin(a, b); break;
            case kMax: r = fmax(a, b); break;
            case kFmod: r = fmod(a, b); break;
            default: r = a; break;
            }
            st[sp - 1] = r;
        }
        }
    }
    return sp > 0 ? st[sp - 1] : 0.0;
}

/// Host compiler: expression text -> postfix program (throws std::invalid_argument on errors).
class Compiler {
  public:
    static std::vector<Instr> compile(const std::string& text) {
        Compiler c(text);
        c.parse_or();
        c.skip();
        if (c.pos != c.s.size()) c.fail("unexpected '" + c.s.substr(c.pos, 1) + "'");
        if (c.max_depth > kMaxStack) c.fail("expression too deep");
        return c.code;
    }

  private:
    explicit Compiler(const std::string& t) : s(t) {}
    std::string s;
    size_t pos = 0;
    std::vector<Instr> code;
    int depth = 0, max_depth = 0;

    [[noreturn]] void fail(const std::string& m) const {
        throw std::invalid_argument("expression \"" + s + "\": " + m + " at position " + std::to_string(pos));
    }
    void emit(int op, double v = 0.0) {
        code.push_back({op, v});
        if (op == kConst || op == kX || op == kY || op == kZ)
            ++depth;
        else if (op == kIf)
            depth -= 2;
        else if (op >= kAdd && op != kNeg && !(op >= kSin && op <= kHeaviside))
            --depth;
        if (depth > max_depth) max_depth = depth;
    }
    void skip() {
        while (pos < s.size() && std::isspace(static_cast<unsigned char>(s[pos]))) ++pos;
    }
    bool eat(const char* tok) {
        skip();
        const size_t n = std::char_traits<char>::length(tok);
        if (s.compare(pos, n, tok) != 0) return false;
        // word operators must not run into an identifier
        if (std::isalpha(static_cast<unsigned char>(tok[0])) && pos + n < s.size() &&
            (std::isalnum(static_cast<unsigned char>(s[pos + n])) || s[pos + n] == '_'))
            return false;
        pos += n;
        return true;
    }
    void parse_or() {
        parse_and();
        while (eat("||") || eat("or")) {
            parse_and();
            emit(kOr);
        }
    }
    void parse_and() {
        parse_cmp();
        while (eat("&&") || eat("and")) {
            parse_cmp();
            emit(kAnd);
        }
    }
    void parse_cmp() {
        parse_add();
        int op = -1;
        if (eat("<=")) op = kLe;
        else if (eat(">=")) op = kGe;
        else if (eat("==")) op = kEq;
        else if (eat("!=")) op = kNe;
        else if (eat("<")) op = kLt;
        else if (eat(">")) op = kGt;
        if (op >= 0) {
            parse_add();
            emit(op);
        }
    }
    void parse_add() {
        parse_mul();
        for (;;) {
            if (eat("+")) {
                parse_mul();
                emit(kAdd);
            } else if (eat("-")) {
                parse_mul();
                emit(kSub);
            } else {
                return;
            }
        }
    }
    void parse_mul() {
        parse_unary();
        for (;;) {
            skip();
            if (s.compare(pos, 2, "**") == 0) return; // power, handled below the unary level
            if (eat("*")) {
                parse_unary();
                emit(kMul);
            } else if (eat("/")) {
                parse_unary();
                emit(kDiv);
            } else {
                return;
            }
        }
    }
    void parse_unary() {
        if (eat("-")) {
            parse_unary();
            emit(kNeg);
        } else if (eat("+")) {
            parse_unary();
        } else {
            parse_power();
        }
    }
    void parse_power() {
        parse_primary();
        if (eat("**") || eat("^")) {
            parse_unary();
            emit(kPow);
        }
    }
    void parse_primary() {
        skip();
        if (pos >= s.size()) fail("unexpected end");
        const char ch = s[pos];
        if (ch == '(') {
            ++pos;
            parse_or();
            if (!eat(")")) fail("missing ')'");
            return;
        }
        if (std::isdigit(static_cast<unsigned char>(ch)) || ch == '.') {
            size_t used = 0;
            double v = 0.0;
            try {
                v = std::stod(s.substr(pos), &used);
            } catch (const std::exception&) {
                fail("bad number");
            }
            pos += used;
            emit(kConst, v);
            return;
        }
        if (std::isalpha(static_cast<unsigned char>(ch)) || ch == '_') {
            size_t e = pos;
            while (e < s.size() && (std::isalnum(static_cast<unsigned char>(s[e])) || s[e] == '_')) ++e;
            const std::string name = s.substr(pos, e - pos);
            pos = e;
            if (name == "x") return emit(kX);
            if (name == "y") return emit(kY);
            if (name == "z") return emit(kZ);
            if (name == "pi") return emit(kConst, 3.14159265358979323846);
            static const struct {
                const char* name;
                int op, nargs;
            } fns[] = {{"sin", kSin, 1},     {"cos", kCos, 1},     {"tan", kTan, 1},       {"asin", kAsin, 1},
                       {"acos", kAcos, 1},   {"atan", kAtan, 1},   {"sinh", kSinh, 1},     {"cosh", kCosh, 1},
                       {"tanh", kTanh, 1},   {"exp", kExp, 1},     {"log", kLog, 1},       {"log10", kLog10, 1},
                       {"sqrt", kSqrt, 1},   {"abs", kAbs, 1},     {"fabs", kAbs, 1},      {"floor", kFloor, 1},
                       {"ceil", kCeil, 1},   {"erf", kErf, 1},     {"heaviside", kHeaviside, 1},
                       {"pow", kPow, 2},     {"atan2", kAtan2, 2}, {"min", kMin, 2},       {"max", kMax, 2},
                       {"fmod", kFmod, 2},   {"if", kIf, 3}};
            for (const auto& f : fns) {
                if (name != f.name) continue;
                if (!eat("(")) fail("missing '(' after " + name);
                for (int a = 0; a < f.nargs; ++a) {
                    if (a > 0 && !eat(",")) fail(name + " takes " + std::to_string(f.nargs) + " arguments");
                    parse_or();
                }
                if (!eat(")")) fail("missing ')' after the arguments of " + name);
                return emit(f.op);
            }
            fail("unknown name '" + name + "'");
        }
        fail("unexpected '" + std::string(1, ch) + "'");
    }
};

} // namespace expr
} // namespace treesap
