// expr.cpp — parser and bytecode compiler for AdditionalCompute expressions.
//
// Grammar (source/granite/TrajectoryIntegrator.cpp:10-26), parsed as a PEG: ordered
// choice commits to the first alternative that matches; spaces and tabs are skipped at the
// start and after every literal or token; the whole input must be consumed.
//   Expression  <- Primary (Operator Primary)*       precedence: + - (left) below * / (left)
//   Primary     <- '(' Expression ')' / Function / Register / OldRegister / Identifier / Constant
//   Function    <- sqrt|exp|ln|sin|cos|tan|asin|acos|atan '(' E ')' / 'atan2' '(' E ',' E ')'
//   Register    <- x | y | z | cv | u | v | w            (no word boundary)
//   OldRegister <- f0..f7 | c0..c3                        (rejected, cpp:110-114)
//   Identifier  <- [_a-zA-Z][a-zA-Z0-9_]*                 (bound to volumes / constants)
//   Constant    <- -?[0-9]+.[0-9]+ / -?[0-9]+             (float32, correctly rounded)
// After parsing: identifiers are bound (cpp:744-768) and tokens are checked against the
// enabled features in the reference's order (TrajectoryIntegrator.tpp:661-696).
#include "expr.h"

#include <cmath>
#include <cstdlib>
#include <memory>
#include <stdexcept>

namespace granite_b200 {
namespace {

// Node kinds use the reference's ASTNodeType values (Language.hpp:17-73).
enum Kind : int {
    K_NONE = 0, K_X = 1, K_Y = 2, K_Z = 3, K_CV = 4, K_F0 = 5, K_C0 = 13, K_CONST = 17,
    K_ADD = 18, K_MUL = 19, K_SUB = 20, K_DIV = 21, K_FN0 = 22, K_ATAN2 = 31, K_IDENT = 32,
    K_U = 33, K_V = 34, K_W = 35
};

struct Ast {
    int kind = K_NONE;
    float value = 0.f;
    std::string id;
    std::unique_ptr<Ast> l, r;
};
using AstP = std::unique_ptr<Ast>;

struct UserError : std::runtime_error {
    using std::runtime_error::runtime_error;
};

std::string user_msg(const std::string &m) { return "ERROR < USER INPUT | " + m + " >"; }

class Parser {
  public:
    explicit Parser(const std::string &s) : s_(s) {}

    AstP parse_all() {
        size_t pos = ws(0);
        AstP e = expression(pos);
        if (!e || pos != s_.size()) {
            size_t col = e ? pos + 1 : 1;
            throw UserError(user_msg("syntax error at column " + std::to_string(col) +
                                     " ( LINE: 1 COLUMN: " + std::to_string(col) + ")"));
        }
        return e;
    }

  private:
    const std::string &s_;

    size_t ws(size_t i) const {
        while (i < s_.size() && (s_[i] == ' ' || s_[i] == '\t')) ++i;
        return i;
    }
    bool lit(size_t &i, const char *w) const {
        size_t n = std::char_traits<char>::length(w);
        if (s_.compare(i, n, w) == 0) {
            i = ws(i + n);
            return true;
        }
        return false;
    }
    static bool is_alpha(char c) { return (c >= 'a' && c <= 'z') || (c >= 'A' && c <= 'Z'); }
    static bool is_digit(char c) { return c >= '0' && c <= '9'; }

    static int prec(char op) { return (op == '+' || op == '-') ? 1 : 2; }
    static int kind_of(char op) {
        switch (op) {
            case '+': return K_ADD;
            case '-': return K_SUB;
            case '*': return K_MUL;
            default: return K_DIV;
        }
    }

    AstP expression(size_t &i) {
        size_t p = i;
        AstP first = primary(p);
        if (!first) return nullptr;
        std::vector<AstP> operands;
        std::vector<char> ops;
        operands.push_back(std::move(first));
        for (;;) {
            if (p < s_.size() && (s_[p] == '+' || s_[p] == '-' || s_[p] == '*' || s_[p] == '/')) {
                size_t q = ws(p + 1);
                AstP nxt = primary(q);
                if (!nxt) break;
                ops.push_back(s_[p]);
                operands.push_back(std::move(nxt));
                p = q;
            } else {
                break;
            }
        }
        size_t idx = 0;
        AstP lhs = std::move(operands[0]);
        AstP tree = climb(std::move(lhs), operands, ops, idx, 1);
        i = p;
        return tree;
    }

    // Precedence climbing; both levels associate to the left.
    AstP climb(AstP lhs, std::vector<AstP> &operands, const std::vector<char> &ops, size_t &idx,
               int min_prec) {
        while (idx < ops.size() && prec(ops[idx]) >= min_prec) {
            char op = ops[idx];
            AstP rhs = std::move(operands[idx + 1]);
            ++idx;
            while (idx < ops.size() && prec(ops[idx]) > prec(op))
                rhs = climb(std::move(rhs), operands, ops, idx, prec(op) + 1);
            auto node = std::make_unique<Ast>();
            node->kind = kind_of(op);
            node->l = std::move(lhs);
            node->r = std::move(rhs);
            lhs = std::move(node);
        }
        return lhs;
    }

    AstP primary(size_t &i) {
        size_t p = i;
        if (lit(p, "(")) {
            AstP e = expression(p);
            if (e && lit(p, ")")) {
                i = p;
                return e;
            }
        }
        p = i;
        if (AstP f = function(p)) {
            i = p;
            return f;
        }
        static const std::pair<const char *, int> regs[] = {
            {"x", K_X}, {"y", K_Y}, {"z", K_Z}, {"cv", K_CV}, {"u", K_U}, {"v", K_V}, {"w", K_W}};
        for (const auto &r : regs) {
            p = i;
            if (lit(p, r.first)) {
                auto n = std::make_unique<Ast>();
                n->kind = r.second;
                i = p;
                return n;
            }
        }
        static const char *old_regs[] = {"f0", "f1", "f2", "f3", "f4", "f5", "f6", "f7",
                                         "c0", "c1", "c2", "c3"};
        for (const char *o : old_regs)
            if (s_.compare(i, 2, o) == 0)
                throw UserError(user_msg(std::string("Identifier '") + o +
                                         "' is no longer allowed, see documentation for more information."));
        if (i < s_.size() && (s_[i] == '_' || is_alpha(s_[i]))) {
            size_t j = i + 1;
            while (j < s_.size() && (s_[j] == '_' || is_alpha(s_[j]) || is_digit(s_[j]))) ++j;
            auto n = std::make_unique<Ast>();
            n->kind = K_IDENT;
            n->id = s_.substr(i, j - i);
            i = ws(j);
            return n;
        }
        return constant(i);
    }

    AstP function(size_t &i) {
        static const char *names[] = {"sqrt", "exp", "ln", "sin", "cos", "tan",
                                      "asin", "acos", "atan", "atan2"};
        for (int k = 0; k < 10; ++k) {
            size_t p = i;
            if (!lit(p, names[k]) || !lit(p, "(")) continue;
            AstP a = expression(p);
            if (!a) continue;
            AstP b;
            if (k == 9) {
                if (!lit(p, ",")) continue;
                b = expression(p);
                if (!b) continue;
            }
            if (!lit(p, ")")) continue;
            auto n = std::make_unique<Ast>();
            n->kind = K_FN0 + k;
            n->l = std::move(a);
            n->r = std::move(b);
            i = p;
            return n;
        }
        return nullptr;
    }

    AstP constant(size_t &i) {
        auto digits = [&](size_t k) -> size_t {
            size_t st = k;
            while (k < s_.size() && is_digit(s_[k])) ++k;
            return k > st ? k : std::string::npos;
        };
        for (int decimal = 1; decimal >= 0; --decimal) {
            size_t k = i;
            if (k < s_.size() && s_[k] == '-') ++k;
            k = digits(k);
            if (k == std::string::npos) continue;
            if (decimal) {
                if (k >= s_.size() || s_[k] != '.') continue;
                size_t k2 = digits(k + 1);
                if (k2 == std::string::npos) continue;
                k = k2;
            }
            auto n = std::make_unique<Ast>();
            n->kind = K_CONST;
            std::string tok = s_.substr(i, k - i);
            n->value = std::strtof(tok.c_str(), nullptr);
            i = ws(k);
            return n;
        }
        return nullptr;
    }
};

void bind(Ast *n, const std::vector<std::string> &vol, const std::vector<std::string> &con) {
    if (n->kind == K_IDENT) {
        int kind = -1;
        for (size_t k = 0; k < vol.size() && k < 8; ++k)
            if (vol[k] == n->id) kind = K_F0 + static_cast<int>(k);
        for (size_t k = 0; k < con.size() && k < 4; ++k)
            if (con[k] == n->id) kind = K_C0 + static_cast<int>(k);
        if (kind < 0) throw UserError(user_msg("Invalid identifier '" + n->id + "'."));
        n->kind = kind;
        n->l.reset();
        n->r.reset();
    }
    if (n->l) bind(n->l.get(), vol, con);
    if (n->r) bind(n->r.get(), vol, con);
}

bool contains(const Ast *n, int kind) {
    if (!n) return false;
    return n->kind == kind || contains(n->l.get(), kind) || contains(n->r.get(), kind);
}

// Registers needed to evaluate a subtree when the deeper operand goes first.
int need(const Ast *n) {
    if (!n->l && !n->r) return 1;
    if (n->l && !n->r) return need(n->l.get());
    int a = need(n->l.get()), b = need(n->r.get());
    return a == b ? a + 1 : (a > b ? a : b);
}

void emit(const Ast *n, std::vector<Instr> &code) {
    const int k = n->kind;
    if (k >= K_X && k <= K_C0 + 3 && k != K_CONST) {
        int slot = k == K_X ? REF_X : k == K_Y ? REF_Y : k == K_Z ? REF_Z : k == K_CV ? REF_CV
                 : (k >= K_F0 && k < K_F0 + 8) ? REF_F0 + (k - K_F0) : REF_C0 + (k - K_C0);
        code.push_back({OP_REF, static_cast<int16_t>(slot), 0.f});
        return;
    }
    if (k == K_U || k == K_V || k == K_W) {
        code.push_back({OP_REF, static_cast<int16_t>(REF_U + (k - K_U)), 0.f});
        return;
    }
    if (k == K_CONST) {
        code.push_back({OP_CONST, 0, n->value});
        return;
    }
    if (k >= K_FN0 && k < K_ATAN2) {
        emit(n->l.get(), code);
        code.push_back({static_cast<int16_t>(OP_SQRT + (k - K_FN0)), 0, 0.f});
        return;
    }
    if (k == K_ADD || k == K_SUB || k == K_MUL || k == K_DIV || k == K_ATAN2) {
        const bool right_first = need(n->r.get()) > need(n->l.get());
        if (right_first) {
            emit(n->r.get(), code);
            emit(n->l.get(), code);
        } else {
            emit(n->l.get(), code);
            emit(n->r.get(), code);
        }
        int16_t op = 0;
        switch (k) {
            case K_ADD: op = OP_ADD; break;   // commutative in IEEE arithmetic
            case K_MUL: op = OP_MUL; break;
            case K_SUB: op = right_first ? OP_RSUB : OP_SUB; break;
            case K_DIV: op = right_first ? OP_RDIV : OP_DIV; break;
            default: op = right_first ? OP_RATAN2 : OP_ATAN2; break;
        }
        code.push_back({op, 0, 0.f});
        return;
    }
    // None / unknown evaluate to 0 (TrajectoryIntegrator.hpp:625)
    code.push_back({OP_CONST, 0, 0.f});
}

}  // namespace

bool compile_expression(const std::string &code, const std::vector<std::string> &volume_names,
                        const std::vector<std::string> &constant_names, int dim,
                        int curvature_mode, Program &out, std::string &error) {
    try {
        Parser parser(code);
        AstP ast = parser.parse_all();
        bind(ast.get(), volume_names, constant_names);
        const size_t nv = volume_names.size() < 8 ? volume_names.size() : 8;
        const size_t nc = constant_names.size() < 4 ? constant_names.size() : 4;
        if (dim == 2 && contains(ast.get(), K_Z))
            throw UserError(user_msg("Compute code contains undefinded token 'z'"));
        if (dim == 2 && contains(ast.get(), K_W))
            throw UserError(user_msg("Compute code contains undefinded token 'w'"));
        for (int k = 7; k >= 0; --k)
            if (nv < static_cast<size_t>(k + 1) && contains(ast.get(), K_F0 + k))
                throw UserError(user_msg("Compute code contains undefinded token 'f" + std::to_string(k) + "'"));
        for (int k = 0; k < 4; ++k)
            if (nc < static_cast<size_t>(k + 1) && contains(ast.get(), K_C0 + k))
                throw UserError(user_msg("Compute code contains undefinded token 'c" + std::to_string(k) + "'"));
        if (curvature_mode != 3 && contains(ast.get(), K_CV))
            throw UserError(user_msg("Compute code contains undefinded token 'cv'"));
        const int depth = need(ast.get());
        if (depth > GR_EXPR_MAX_STACK)
            throw UserError(user_msg("Compute code '" + code + "' needs an operand stack deeper than " +
                                     std::to_string(GR_EXPR_MAX_STACK)));
        std::vector<Instr> prog;
        emit(ast.get(), prog);
        if (prog.size() > static_cast<size_t>(GR_EXPR_MAX_CODE))
            throw UserError(user_msg("Compute code '" + code + "' is longer than " +
                                     std::to_string(GR_EXPR_MAX_CODE) + " operations"));
        out.len = static_cast<int32_t>(prog.size());
        out.depth = depth;
        for (size_t i = 0; i < prog.size(); ++i) out.code[i] = prog[i];
        return true;
    } catch (const UserError &e) {
        error = e.what();
        return false;
    }
}

float evaluate(const Program &p, const float *ref) {
    float st[GR_EXPR_MAX_STACK + 1];
    int sp = 0;
    for (int k = 0; k < p.len; ++k) {
        const Instr &in = p.code[k];
        switch (in.op) {
            case OP_REF: st[sp++] = ref[in.arg]; break;
            case OP_CONST: st[sp++] = in.value; break;
            case OP_ADD: st[sp - 2] = st[sp - 2] + st[sp - 1]; --sp; break;
            case OP_SUB: st[sp - 2] = st[sp - 2] - st[sp - 1]; --sp; break;
            case OP_MUL: st[sp - 2] = st[sp - 2] * st[sp - 1]; --sp; break;
            case OP_DIV: st[sp - 2] = st[sp - 2] / st[sp - 1]; --sp; break;
            case OP_RSUB: st[sp - 2] = st[sp - 1] - st[sp - 2]; --sp; break;
            case OP_RDIV: st[sp - 2] = st[sp - 1] / st[sp - 2]; --sp; break;
            case OP_ATAN2: st[sp - 2] = std::atan2(st[sp - 2], st[sp - 1]); --sp; break;
            case OP_RATAN2: st[sp - 2] = std::atan2(st[sp - 1], st[sp - 2]); --sp; break;
            case OP_SQRT: st[sp - 1] = std::sqrt(st[sp - 1]); break;
            case OP_EXP: st[sp - 1] = std::exp(st[sp - 1]); break;
            case OP_LOG: st[sp - 1] = std::log(st[sp - 1]); break;
            case OP_SIN: st[sp - 1] = std::sin(st[sp - 1]); break;
            case OP_COS: st[sp - 1] = std::cos(st[sp - 1]); break;
            case OP_TAN: st[sp - 1] = std::tan(st[sp - 1]); break;
            case OP_ASIN: st[sp - 1] = std::asin(st[sp - 1]); break;
            case OP_ACOS: st[sp - 1] = std::acos(st[sp - 1]); break;
            case OP_ATAN: st[sp - 1] = std::atan(st[sp - 1]); break;
            default: break;
        }
    }
    return sp > 0 ? st[sp - 1] : 0.f;
}

}  // namespace granite_b200
