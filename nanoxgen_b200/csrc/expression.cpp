// expression.cpp -- host compiler for XGen scalar expressions.
//
// Produces the SSA program that the device evaluator (classic.cu) runs for
// every root.  The language, the compiled program and the error texts follow
// the reference compiler:
//   source normalisation        src/xgen_expression.cpp:50-118
//   tokens                      src/xgen_expression.cpp:120-223
//   grammar / SSA emission      src/xgen_expression.cpp:225-557
//   float program conversion    src/xgen_expression.cpp:783-818
//   seeds and the SeExpr hash   src/xgen_expression.cpp:614-737
//   Classic rewrites            src/xgen_classic_runtime.cpp:88-347
// Compiled with -ffp-contract=off so the double-precision seed arithmetic
// rounds exactly as the reference's does.
#include "nxg_internal.h"
#include "nxg_classic.h"
#include "expression.h"

#include <charconv>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <limits>
#include <new>
#include <stdexcept>
#include <string>
#include <unordered_map>
#include <vector>

namespace nxg {
namespace {

// SeExpr's byte permutation (the hash's final mixing step).  Generated by
// make_permutation_table.py from the reference's own hash function.
constexpr uint8_t kPermutation[256] = {
#include "seexpr_permutation.inc"
};

struct CompileError {
    std::string text;
};

[[noreturn]] void fail(std::string text) { throw CompileError{std::move(text)}; }

[[noreturn]] void syntax(size_t offset, const std::string &what) {
    fail("XGen scalar expression error at byte " + std::to_string(offset) + ": " + what);
}

// ----------------------------------------------------------------- hashing

uint32_t seexpr_component(double argument) {
    int exponent = 0;
    const double fraction = std::frexp(argument * 8.539734222673566, &exponent);
    return static_cast<uint32_t>(fraction * 4294967295.0) ^ static_cast<uint32_t>(exponent);
}

uint32_t hash_finish(uint32_t s) {
    s ^= s >> 11u;
    s ^= (s << 7u) & 0x9d2c5680u;
    s ^= (s << 15u) & 0xefc60000u;
    s ^= s >> 18u;
    const uint32_t b3 = kPermutation[s & 0xffu];
    const uint32_t b2 = kPermutation[((s >> 8u) + b3) & 0xffu];
    const uint32_t b1 = kPermutation[((s >> 16u) + b2) & 0xffu];
    const uint32_t b0 = kPermutation[((s >> 24u) + b1) & 0xffu];
    return b0 | (b1 << 8u) | (b2 << 16u) | (b3 << 24u);
}

double seexpr_hash(const double *arguments, size_t count) {
    uint32_t state = 0u;
    for (size_t i = 0; i < count; ++i) { state = state * 1664525u + seexpr_component(arguments[i]) + 1013904223u; }
    return static_cast<double>(hash_finish(state)) * (1.0 / 4294967295.0);
}

uint32_t string_seed(const std::string &text) {
    uint32_t hash = 0u;
    for (const unsigned char c : text) {
        hash = (hash << 4u) + c;
        const uint32_t high = hash & 0xf0000000u;
        if (high != 0u) {
            hash ^= high >> 24u;
            hash &= ~high;
        }
    }
    return hash % 211u;
}

// ----------------------------------------------------------------- program

struct Instruction {
    uint8_t op;
    uint32_t operand_offset;
    uint16_t operand_count;
    uint32_t auxiliary;
    double immediate;
};

struct RampPoint {
    double position;
    double value;
    uint8_t interpolation;
};

struct Program {
    std::vector<Instruction> instructions;
    std::vector<uint32_t> operands;
    std::vector<std::string> inputs;
    std::vector<RampPoint> ramp_points;
    std::vector<ExprRamp> ramps;
    uint32_t result = 0;
    uint32_t expression_seed = 0;
    uint32_t random_call_count = 0;
};

// Limits of the reference's XgenExpressionCompileOptions defaults.
constexpr size_t kMaxSourceBytes = 1024u * 1024u;
constexpr size_t kMaxTokens = 100000u;
constexpr size_t kMaxInstructions = 100000u;
constexpr size_t kMaxLocals = 4096u;
constexpr size_t kMaxRampPoints = 4096u;

// ------------------------------------------------------------ normalising

bool continues_line(char c) {
    switch (c) {
        case '+': case '-': case '*': case '/': case '<': case '>': case '=': case '!':
        case '&': case '|': case '?': case ':': case ',': case '(':
            return true;
        default:
            return false;
    }
}

// '#' comments end at a newline, which becomes ';'.  A newline then joins the
// lines (a space) when the text before it ends, or the text after it starts,
// with an operator; otherwise it separates statements (';').
std::string normalise(const std::string &source) {
    if (source.size() > kMaxSourceBytes) { fail("XGen scalar expression source byte limit exceeded"); }
    if (source.find('\0') != std::string::npos) { fail("XGen scalar expression contains a NUL byte"); }
    std::string stripped;
    stripped.reserve(source.size());
    bool in_comment = false;
    for (size_t i = 0; i < source.size(); ++i) {
        char c = source[i];
        if (c == '\\' && i + 1 < source.size() && source[i + 1] == 'n') {
            c = '\n';
            ++i;
        }
        if (in_comment) {
            if (c == '\n' || c == '\r') {
                in_comment = false;
                stripped.push_back(';');
            }
        } else if (c == '#') {
            in_comment = true;
        } else {
            stripped.push_back(c);
        }
    }
    std::string joined;
    joined.reserve(stripped.size());
    for (size_t i = 0; i < stripped.size(); ++i) {
        const char c = stripped[i];
        if (c != '\n' && c != '\r') {
            joined.push_back(c);
            continue;
        }
        size_t before = joined.size();
        while (before > 0 && (joined[before - 1] == ' ' || joined[before - 1] == '\t')) { --before; }
        size_t after = i + 1;
        while (after < stripped.size() &&
               (stripped[after] == ' ' || stripped[after] == '\t' || stripped[after] == '\n' ||
                stripped[after] == '\r')) {
            ++after;
        }
        const bool with_previous = before > 0 && continues_line(joined[before - 1]);
        const bool with_next =
            after < stripped.size() && (continues_line(stripped[after]) || stripped[after] == ')');
        joined.push_back(with_previous || with_next ? ' ' : ';');
    }
    return joined;
}

// ------------------------------------------------------------------ tokens

enum class Tok : uint8_t {
    End, Number, Variable, Identifier, String, Semicolon, Comma, LParen, RParen, Question, Colon,
    Assign, Plus, Minus, Star, Slash, Bang, Arrow, Less, LessEqual, Greater, GreaterEqual, Equal,
    NotEqual, And, Or
};

struct Token {
    Tok kind = Tok::End;
    std::string text;
    double number = 0.0;
    size_t offset = 0;
};

bool ident_start(char c) { return (c >= 'a' && c <= 'z') || (c >= 'A' && c <= 'Z') || c == '_'; }
bool ident_part(char c) { return ident_start(c) || (c >= '0' && c <= '9'); }

std::vector<Token> lex(const std::string &s) {
    std::vector<Token> out;
    const auto push = [&out](Tok kind, size_t offset, std::string text = {}, double number = 0.0) {
        if (out.size() >= kMaxTokens) { fail("XGen scalar expression token limit exceeded"); }
        out.push_back(Token{kind, std::move(text), number, offset});
    };
    size_t i = 0;
    while (i < s.size()) {
        const char c = s[i];
        if (c == ' ' || c == '\t' || c == '\f' || c == '\v') {
            ++i;
            continue;
        }
        const bool digit = c >= '0' && c <= '9';
        if (digit || (c == '.' && i + 1 < s.size() && s[i + 1] >= '0' && s[i + 1] <= '9')) {
            const char *begin = s.c_str() + i;
            char *end = nullptr;
            const double value = std::strtod(begin, &end);
            const size_t used = static_cast<size_t>(end - begin);
            if (used == 0 || !std::isfinite(value)) { syntax(i, "invalid or non-finite numeric literal"); }
            push(Tok::Number, i, {}, value);
            i += used;
            continue;
        }
        if (c == '$') {
            const size_t at = i++;
            if (i >= s.size() || !ident_start(s[i])) { syntax(at, "expected a variable name after '$'"); }
            const size_t name = i++;
            while (i < s.size() && ident_part(s[i])) { ++i; }
            push(Tok::Variable, at, s.substr(name, i - name));
            continue;
        }
        if (ident_start(c)) {
            const size_t at = i++;
            while (i < s.size() && ident_part(s[i])) { ++i; }
            push(Tok::Identifier, at, s.substr(at, i - at));
            continue;
        }
        if (c == '\'' || c == '"') {
            const size_t at = i++;
            std::string text;
            while (i < s.size() && s[i] != c) {
                if (s[i] == '\\' && i + 1 < s.size()) { ++i; }
                text.push_back(s[i++]);
            }
            if (i == s.size()) { syntax(at, "unterminated string literal"); }
            ++i;
            push(Tok::String, at, std::move(text));
            continue;
        }
        const auto pair = [&](char second, Tok both, Tok single) {
            if (i + 1 < s.size() && s[i + 1] == second) {
                push(both, i);
                i += 2;
            } else {
                push(single, i);
                ++i;
            }
        };
        switch (c) {
            case ';': push(Tok::Semicolon, i++); break;
            case ',': push(Tok::Comma, i++); break;
            case '(': push(Tok::LParen, i++); break;
            case ')': push(Tok::RParen, i++); break;
            case '?': push(Tok::Question, i++); break;
            case ':': push(Tok::Colon, i++); break;
            case '+': push(Tok::Plus, i++); break;
            case '*': push(Tok::Star, i++); break;
            case '/': push(Tok::Slash, i++); break;
            case '-': pair('>', Tok::Arrow, Tok::Minus); break;
            case '=': pair('=', Tok::Equal, Tok::Assign); break;
            case '!': pair('=', Tok::NotEqual, Tok::Bang); break;
            case '<': pair('=', Tok::LessEqual, Tok::Less); break;
            case '>': pair('=', Tok::GreaterEqual, Tok::Greater); break;
            case '&':
                if (i + 1 >= s.size() || s[i + 1] != '&') { syntax(i, "single '&' is unsupported; use '&&'"); }
                push(Tok::And, i);
                i += 2;
                break;
            case '|':
                if (i + 1 >= s.size() || s[i + 1] != '|') { syntax(i, "single '|' is unsupported; use '||'"); }
                push(Tok::Or, i);
                i += 2;
                break;
            default:
                syntax(i, "unsupported character");
        }
    }
    push(Tok::End, s.size());
    return out;
}

// ------------------------------------------------------------------ parser

// Recursive descent, lowest precedence first: ?: (right associative), ||,
// &&, == !=, < <= > >=, + -, * /, prefix + - !, postfix ->method(...).
// Every value is an SSA instruction index; locals alias earlier values.
class Parser {
public:
    Parser(std::vector<Token> tokens, const std::string &name, const std::string &type)
        : tokens_(std::move(tokens)) {
        program_.expression_seed = string_seed(name + type);
    }

    Program run() {
        bool any = false;
        while (peek().kind != Tok::End) {
            while (accept(Tok::Semicolon)) {}
            if (peek().kind == Tok::End) { break; }
            if ((peek().kind == Tok::Variable || peek().kind == Tok::Identifier) && peek(1).kind == Tok::Assign) {
                const Token target = take();
                take();
                const uint32_t value = expression();
                if (locals_.find(target.text) == locals_.end() && locals_.size() >= kMaxLocals) {
                    fail("XGen scalar expression local limit exceeded");
                }
                locals_[target.text] = value;
                program_.result = value;
            } else {
                program_.result = expression();
            }
            any = true;
            if (peek().kind != Tok::Semicolon && peek().kind != Tok::End) {
                syntax(peek().offset, "expected ';' after expression");
            }
        }
        if (!any) { syntax(0, "expression is empty"); }
        return std::move(program_);
    }

private:
    const Token &peek(size_t ahead = 0) const {
        const size_t at = cursor_ + ahead;
        return tokens_[at < tokens_.size() ? at : tokens_.size() - 1];
    }
    Token take() { return tokens_[cursor_++]; }
    bool accept(Tok kind) {
        if (peek().kind != kind) { return false; }
        ++cursor_;
        return true;
    }
    void expect(Tok kind, const char *what) {
        if (!accept(kind)) { syntax(peek().offset, what); }
    }

    uint32_t emit(ExprOp op, const std::vector<uint32_t> &args = {}, double immediate = 0.0, uint32_t aux = 0) {
        if (program_.instructions.size() >= kMaxInstructions) {
            fail("XGen scalar expression instruction limit exceeded");
        }
        if (args.size() > std::numeric_limits<uint16_t>::max()) {
            fail("XGen scalar expression operand limit exceeded");
        }
        const size_t offset = program_.operands.size();
        if (offset > std::numeric_limits<uint32_t>::max()) {
            fail("XGen scalar expression operand storage exceeded");
        }
        program_.operands.insert(program_.operands.end(), args.begin(), args.end());
        program_.instructions.push_back(Instruction{static_cast<uint8_t>(op), static_cast<uint32_t>(offset),
                                                    static_cast<uint16_t>(args.size()), aux, immediate});
        return static_cast<uint32_t>(program_.instructions.size() - 1);
    }

    uint32_t expression() { return conditional(); }

    uint32_t conditional() {
        const uint32_t test = either();
        if (!accept(Tok::Question)) { return test; }
        const uint32_t yes = expression();
        expect(Tok::Colon, "expected ':' in conditional expression");
        const uint32_t no = conditional();
        return emit(kOpSelect, {test, yes, no});
    }

    uint32_t either() {
        uint32_t v = both();
        while (accept(Tok::Or)) { v = emit(kOpLogicalOr, {v, both()}); }
        return v;
    }

    uint32_t both() {
        uint32_t v = equality();
        while (accept(Tok::And)) { v = emit(kOpLogicalAnd, {v, equality()}); }
        return v;
    }

    uint32_t equality() {
        uint32_t v = relation();
        for (;;) {
            if (accept(Tok::Equal)) {
                v = emit(kOpEqual, {v, relation()});
            } else if (accept(Tok::NotEqual)) {
                v = emit(kOpNotEqual, {v, relation()});
            } else {
                return v;
            }
        }
    }

    uint32_t relation() {
        uint32_t v = sum();
        for (;;) {
            ExprOp op;
            if (accept(Tok::Less)) {
                op = kOpLess;
            } else if (accept(Tok::LessEqual)) {
                op = kOpLessEqual;
            } else if (accept(Tok::Greater)) {
                op = kOpGreater;
            } else if (accept(Tok::GreaterEqual)) {
                op = kOpGreaterEqual;
            } else {
                return v;
            }
            v = emit(op, {v, sum()});
        }
    }

    uint32_t sum() {
        uint32_t v = product();
        for (;;) {
            if (accept(Tok::Plus)) {
                v = emit(kOpAdd, {v, product()});
            } else if (accept(Tok::Minus)) {
                v = emit(kOpSubtract, {v, product()});
            } else {
                return v;
            }
        }
    }

    uint32_t product() {
        uint32_t v = unary();
        for (;;) {
            if (accept(Tok::Star)) {
                v = emit(kOpMultiply, {v, unary()});
            } else if (accept(Tok::Slash)) {
                v = emit(kOpDivide, {v, unary()});
            } else {
                return v;
            }
        }
    }

    uint32_t unary() {
        if (accept(Tok::Plus)) { return unary(); }
        if (accept(Tok::Minus)) { return emit(kOpNegate, {unary()}); }
        if (accept(Tok::Bang)) { return emit(kOpLogicalNot, {unary()}); }
        return methods();
    }

    uint32_t methods() {
        uint32_t v = primary();
        while (accept(Tok::Arrow)) {
            if (peek().kind != Tok::Identifier) { syntax(peek().offset, "expected a method name after '->'"); }
            const Token name = take();
            expect(Tok::LParen, "expected '(' after expression method name");
            std::vector<uint32_t> args{v};
            if (!accept(Tok::RParen)) {
                do {
                    args.push_back(expression());
                } while (accept(Tok::Comma));
                expect(Tok::RParen, "expected ')' after expression method arguments");
            }
            v = call(name, args);
        }
        return v;
    }

    double ramp_number(const char *what) {
        double sign = 1.0;
        if (!accept(Tok::Plus) && accept(Tok::Minus)) { sign = -1.0; }
        if (peek().kind != Tok::Number) { syntax(peek().offset, std::string("expected a numeric ramp ") + what); }
        return sign * take().number;
    }

    // rampUI(position, value, interpolation : position, value, interpolation ...)
    uint32_t ramp(const Token &name) {
        const size_t first = program_.ramp_points.size();
        for (;;) {
            const double position = ramp_number("position");
            expect(Tok::Comma, "expected ',' after ramp position");
            const double value = ramp_number("value");
            expect(Tok::Comma, "expected ',' after ramp value");
            const double interpolation = ramp_number("interpolation");
            if (interpolation != std::floor(interpolation) || interpolation < 0.0 || interpolation > 3.0) {
                syntax(name.offset, "ramp interpolation must be an integer in [0, 3]");
            }
            if (position < 0.0 || position > 1.0) { syntax(name.offset, "ramp positions must be in [0, 1]"); }
            if (program_.ramp_points.size() >= kMaxRampPoints) {
                fail("XGen scalar expression ramp point limit exceeded");
            }
            if (program_.ramp_points.size() != first && position <= program_.ramp_points.back().position) {
                syntax(name.offset, "ramp positions must be strictly increasing");
            }
            program_.ramp_points.push_back(RampPoint{position, value, static_cast<uint8_t>(interpolation)});
            if (!accept(Tok::Colon)) { break; }
        }
        expect(Tok::RParen, "expected ')' after rampUI points");
        const size_t count = program_.ramp_points.size() - first;
        if (count == 0 || count > std::numeric_limits<uint16_t>::max() ||
            first > std::numeric_limits<uint32_t>::max()) {
            syntax(name.offset, "ramp point storage limit exceeded");
        }
        const uint32_t index = static_cast<uint32_t>(program_.ramps.size());
        program_.ramps.push_back(ExprRamp{static_cast<uint32_t>(first), static_cast<uint32_t>(count)});
        return emit(kOpRamp, {}, 0.0, index);
    }

    uint32_t primary() {
        if (peek().kind == Tok::Number) { return emit(kOpConstant, {}, take().number); }
        if (peek().kind == Tok::Variable) {
            const Token v = take();
            const auto local = locals_.find(v.text);
            if (local != locals_.end()) { return local->second; }
            uint32_t index = 0;
            while (index < program_.inputs.size() && program_.inputs[index] != v.text) { ++index; }
            if (index == program_.inputs.size()) { program_.inputs.push_back(v.text); }
            return emit(kOpInput, {}, 0.0, index);
        }
        if (accept(Tok::LParen)) {
            const uint32_t v = expression();
            expect(Tok::RParen, "expected ')'");
            return v;
        }
        if (peek().kind == Tok::String) {
            syntax(peek().offset, "string values require an explicit PTEX binding such as map()");
        }
        if (peek().kind != Tok::Identifier) { syntax(peek().offset, "expected a scalar value"); }
        const Token name = take();
        if (name.text == "true") { return emit(kOpConstant, {}, 1.0); }
        if (name.text == "false") { return emit(kOpConstant, {}, 0.0); }
        if (!accept(Tok::LParen)) {
            const auto local = locals_.find(name.text);
            if (local != locals_.end()) { return local->second; }
            syntax(name.offset, "bare identifier is unsupported: " + name.text);
        }
        if (name.text == "rampUI") { return ramp(name); }
        std::vector<uint32_t> args;
        if (!accept(Tok::RParen)) {
            do {
                args.push_back(expression());
            } while (accept(Tok::Comma));
            expect(Tok::RParen, "expected ')' after function arguments");
        }
        return call(name, args);
    }

    uint32_t call(const Token &name, const std::vector<uint32_t> &args) {
        const auto arity = [&](size_t n) {
            if (args.size() != n) {
                syntax(name.offset, name.text + " expects " + std::to_string(n) + " argument(s)");
            }
        };
        const std::string &f = name.text;
        if (f == "hash") {
            if (args.empty()) { syntax(name.offset, "hash expects at least one argument"); }
            return emit(kOpHash, args);
        }
        if (f == "rand") {
            if (args.size() > 3) { syntax(name.offset, "rand expects zero to three arguments"); }
            // Each call site draws its own seed from (expression seed, call number).
            const double site[2] = {static_cast<double>(program_.expression_seed),
                                    static_cast<double>(program_.random_call_count)};
            const double seed = seexpr_hash(site, 2);
            ++program_.random_call_count;
            return emit(kOpRandom, args, seed);
        }
        if (f == "min") { arity(2); return emit(kOpMinimum, args); }
        if (f == "max") { arity(2); return emit(kOpMaximum, args); }
        if (f == "clamp") { arity(3); return emit(kOpClamp, args); }
        if (f == "fit") { arity(5); return emit(kOpFit, args); }
        if (f == "gamma") { arity(2); return emit(kOpGamma, args); }
        if (f == "contrast") { arity(2); return emit(kOpContrast, args); }
        if (f == "smoothstep") { arity(3); return emit(kOpSmoothstep, args); }
        if (f == "map") {
            syntax(name.offset, "map requires an explicit PTEX binding and is not a scalar intrinsic");
        }
        syntax(name.offset, "unsupported function: " + f);
    }

    std::vector<Token> tokens_;
    size_t cursor_ = 0;
    std::unordered_map<std::string, uint32_t> locals_;
    Program program_;
};

// ------------------------------------------------------- Classic rewrites

bool classic_ident(char c) {
    return (c >= 'a' && c <= 'z') || (c >= 'A' && c <= 'Z') || (c >= '0' && c <= '9') || c == '_';
}

// Classic attribute values: '#' comments (outside quotes) are dropped up to
// the end of the line, and the two characters "\n" become a newline.
std::string classic_strip(const std::string &value) {
    std::string out;
    out.reserve(value.size());
    bool quoted = false;
    char quote = 0;
    size_t i = 0;
    while (i < value.size()) {
        const char c = value[i];
        if (!quoted && c == '\\' && i + 1 < value.size() && value[i + 1] == 'n') {
            out.push_back('\n');
            i += 2;
            continue;
        }
        if (!quoted && c == '#') {
            while (i < value.size() && value[i] != '\n') {
                if (value[i] == '\\' && i + 1 < value.size() && value[i + 1] == 'n') {
                    i += 2;
                    out.push_back('\n');
                    break;
                }
                ++i;
            }
            continue;
        }
        out.push_back(c);
        if (quoted) {
            if (c == quote && (i == 0 || value[i - 1] != '\\')) { quoted = false; }
        } else if (c == '\'' || c == '"') {
            quoted = true;
            quote = c;
        }
        ++i;
    }
    return out;
}

bool parse_float(const char *first, const char *last, float &value, const char *&end) {
    const auto r = std::from_chars(first, last, value, std::chars_format::general);
    end = r.ptr;
    return r.ec == std::errc{};
}

bool blank(char c) { return c == ' ' || c == '\t'; }
bool blank_or_newline(char c) { return c == ' ' || c == '\t' || c == '\r' || c == '\n'; }

// The value of the last "$name = <number>" before `before`, if any.
bool constant_assignment(const std::string &s, const std::string &name, size_t before, float &out) {
    const std::string token = "$" + name;
    bool found = false;
    size_t i = 0;
    while (i < before) {
        i = s.find(token, i);
        if (i == std::string::npos || i >= before) { break; }
        size_t c = i + token.size();
        if (c < s.size() && classic_ident(s[c])) {
            i = c;
            continue;
        }
        while (c < before && blank_or_newline(s[c])) { ++c; }
        if (c >= before || s[c] != '=' || (c + 1 < before && s[c + 1] == '=')) {
            i = c;
            continue;
        }
        ++c;
        while (c < before && blank_or_newline(s[c])) { ++c; }
        float sign = 1.0f;
        if (c < before && (s[c] == '+' || s[c] == '-')) {
            if (s[c++] == '-') { sign = -1.0f; }
        }
        float value = 0.0f;
        const char *end = nullptr;
        if (parse_float(s.data() + c, s.data() + before, value, end) && end != s.data() + c &&
            std::isfinite(value)) {
            out = sign * value;
            found = true;
        }
        i = c;
    }
    return found;
}

// noise($Prefg * k) becomes the input $__nxg_pref_noise_<i>, one input per
// distinct frequency (compared bitwise); other noise forms are left alone
// and then fail to compile as unsupported functions.
std::string classic_rewrite(const std::string &source, std::vector<float> &frequencies) {
    for (size_t i = 0; i + 2 < source.size(); ++i) {
        if (source.compare(i, 3, "map") != 0 || (i != 0 && classic_ident(source[i - 1]))) { continue; }
        size_t c = i + 3;
        while (c < source.size() && blank(source[c])) { ++c; }
        if (c < source.size() && source[c] == '(') {
            fail("PTEX map() inputs are not bound by this runtime");
        }
    }
    std::string s = source;
    size_t i = 0;
    for (;;) {
        i = s.find("noise", i);
        if (i == std::string::npos) { break; }
        if ((i != 0 && classic_ident(s[i - 1])) || (i + 5 < s.size() && classic_ident(s[i + 5]))) {
            i += 5;
            continue;
        }
        size_t c = i + 5;
        while (c < s.size() && blank(s[c])) { ++c; }
        if (c >= s.size() || s[c++] != '(') {
            i += 5;
            continue;
        }
        while (c < s.size() && blank(s[c])) { ++c; }
        static const std::string prefg = "$Prefg";
        if (s.compare(c, prefg.size(), prefg) != 0 ||
            (c + prefg.size() < s.size() && classic_ident(s[c + prefg.size()]))) {
            i += 5;
            continue;
        }
        c += prefg.size();
        while (c < s.size() && blank(s[c])) { ++c; }
        if (c >= s.size() || s[c++] != '*') {
            i += 5;
            continue;
        }
        while (c < s.size() && blank(s[c])) { ++c; }
        bool have = false;
        float frequency = 0.0f;
        if (c < s.size() && s[c] == '$') {
            const size_t name = ++c;
            while (c < s.size() && classic_ident(s[c])) { ++c; }
            if (c != name) { have = constant_assignment(s, s.substr(name, c - name), i, frequency); }
        } else {
            float sign = 1.0f;
            if (c < s.size() && (s[c] == '+' || s[c] == '-')) {
                if (s[c++] == '-') { sign = -1.0f; }
            }
            float value = 0.0f;
            const char *end = nullptr;
            if (parse_float(s.data() + c, s.data() + s.size(), value, end) && end != s.data() + c &&
                std::isfinite(value)) {
                frequency = sign * value;
                have = true;
                c = static_cast<size_t>(end - s.data());
            }
        }
        while (c < s.size() && blank(s[c])) { ++c; }
        if (!have || c >= s.size() || s[c++] != ')') {
            i += 5;
            continue;
        }
        uint32_t bits;
        std::memcpy(&bits, &frequency, 4);
        size_t index = 0;
        for (; index < frequencies.size(); ++index) {
            uint32_t other;
            std::memcpy(&other, &frequencies[index], 4);
            if (other == bits) { break; }
        }
        if (index == frequencies.size()) {
            if (frequencies.size() >= 61u) { fail("runtime external input limit exceeded"); }
            frequencies.push_back(frequency);
        }
        const std::string input = "$__nxg_pref_noise_" + std::to_string(index);
        s.replace(i, c - i, input);
        i += input.size();
    }
    return s;
}

} // namespace

// The opaque handle: the float program (the device form's source) and the
// Classic rewrite's noise frequencies.
struct Expression {
    std::vector<ExprInstruction> instructions;
    std::vector<uint32_t> operands;
    std::vector<std::string> inputs;
    std::vector<ExprRampPoint> ramp_points;
    std::vector<ExprRamp> ramps;
    std::vector<float> pref_noise;
    uint32_t result = 0;
    uint32_t expression_seed = 0;
    uint32_t random_call_count = 0;
};

namespace {

Expression to_float_program(const Program &p, std::vector<float> frequencies) {
    Expression e;
    e.instructions.reserve(p.instructions.size());
    for (const Instruction &in : p.instructions) {
        const float immediate = static_cast<float>(in.immediate);
        if (!std::isfinite(immediate)) { fail("XGen expression immediate cannot be represented as float"); }
        const uint32_t aux = in.op == kOpRandom ? seexpr_component(in.immediate) : in.auxiliary;
        e.instructions.push_back(ExprInstruction{in.op, 0, in.operand_count, in.operand_offset, aux, immediate});
    }
    e.operands = p.operands;
    e.inputs = p.inputs;
    for (const RampPoint &rp : p.ramp_points) {
        const float position = static_cast<float>(rp.position);
        const float value = static_cast<float>(rp.value);
        if (!std::isfinite(position) || !std::isfinite(value)) {
            fail("XGen ramp point cannot be represented as float");
        }
        e.ramp_points.push_back(ExprRampPoint{position, value, rp.interpolation});
    }
    e.ramps = p.ramps;
    e.result = p.result;
    e.expression_seed = p.expression_seed;
    e.random_call_count = p.random_call_count;
    e.pref_noise = std::move(frequencies);
    return e;
}

void copy_message(const std::string &text, char *message, size_t capacity) {
    if (message == nullptr || capacity == 0) { return; }
    const size_t n = text.size() < capacity - 1 ? text.size() : capacity - 1;
    std::memcpy(message, text.data(), n);
    message[n] = '\0';
}

uint32_t pack(const Expression &e, DeviceExpression &d) {
    std::memset(&d, 0, sizeof d);
    if (e.instructions.size() > kExprMaxInstructions || e.operands.size() > kExprMaxOperands ||
        e.inputs.size() > kExprMaxInputs || e.ramp_points.size() > kExprMaxRampPoints ||
        e.ramps.size() > kExprMaxRamps) {
        return NXG_ERROR_EXPRESSION_LIMIT;
    }
    d.instruction_count = static_cast<uint32_t>(e.instructions.size());
    d.operand_count = static_cast<uint32_t>(e.operands.size());
    d.input_count = static_cast<uint32_t>(e.inputs.size());
    d.ramp_count = static_cast<uint32_t>(e.ramps.size());
    d.ramp_point_count = static_cast<uint32_t>(e.ramp_points.size());
    d.result = e.result;
    d.present = 1u;
    // The compiler emits well-formed programs; the checks keep every device
    // read inside the packed arrays whatever the handle holds.
    if (e.instructions.empty() || e.result >= e.instructions.size()) { return NXG_ERROR_EXPRESSION_LIMIT; }
    for (size_t i = 0; i < e.instructions.size(); ++i) {
        const ExprInstruction &in = e.instructions[i];
        if (in.op >= kOpCount || uint64_t{in.operand_offset} + in.operand_count > e.operands.size()) {
            return NXG_ERROR_EXPRESSION_LIMIT;
        }
        for (uint32_t k = 0; k < in.operand_count; ++k) {
            if (e.operands[in.operand_offset + k] >= i) { return NXG_ERROR_EXPRESSION_LIMIT; }
        }
        if (in.op == kOpInput && in.auxiliary >= e.inputs.size()) { return NXG_ERROR_EXPRESSION_LIMIT; }
        if (in.op == kOpRamp) {
            if (in.auxiliary >= e.ramps.size()) { return NXG_ERROR_EXPRESSION_LIMIT; }
            const ExprRamp &r = e.ramps[in.auxiliary];
            if (r.point_count == 0 || uint64_t{r.point_offset} + r.point_count > e.ramp_points.size()) {
                return NXG_ERROR_EXPRESSION_LIMIT;
            }
        }
        if (in.op == kOpRandom) { d.uses_random = 1u; }
        d.instructions[i] = in;
    }
    for (size_t i = 0; i < e.operands.size(); ++i) { d.operands[i] = static_cast<uint16_t>(e.operands[i]); }
    for (size_t i = 0; i < e.ramp_points.size(); ++i) { d.ramp_points[i] = e.ramp_points[i]; }
    for (size_t i = 0; i < e.ramps.size(); ++i) { d.ramps[i] = e.ramps[i]; }
    for (size_t i = 0; i < e.inputs.size(); ++i) {
        const std::string &name = e.inputs[i];
        static const std::string noise = "__nxg_pref_noise_";
        if (name.compare(0, noise.size(), noise) == 0) {
            const std::string digits = name.substr(noise.size());
            uint32_t k = 0;
            const auto r = std::from_chars(digits.data(), digits.data() + digits.size(), k);
            if (digits.empty() || r.ec != std::errc{} || r.ptr != digits.data() + digits.size() ||
                k >= e.pref_noise.size()) {
                return NXG_ERROR_EXPRESSION_INPUT;
            }
            d.input_binding[i] = kBindPrefNoise;
            d.input_frequency[i] = e.pref_noise[k];
        } else if (name == "id") {
            d.input_binding[i] = kBindId;
        } else if (name == "u") {
            d.input_binding[i] = kBindU;
        } else if (name == "v") {
            d.input_binding[i] = kBindV;
        } else if (name == "cLength") {
            d.input_binding[i] = kBindCLength;
            d.uses_clength = 1u;
        } else if (name == "cWidth") {
            d.input_binding[i] = kBindCWidth;
        } else {
            return NXG_ERROR_EXPRESSION_INPUT;
        }
    }
    return NXG_ERROR_NONE;
}

} // namespace
} // namespace nxg

struct nxg_expression : nxg::Expression {};

namespace nxg {

uint32_t pack_device_expression(const nxg_expression *e, DeviceExpression &d) { return pack(*e, d); }

} // namespace nxg

using nxg::Expression;

extern "C" {

uint32_t nxg_expression_compile(const char *source, const char *expression_name, const char *object_type,
                                uint32_t flags, nxg_expression **out, char *message, size_t message_capacity) {
    if (source == nullptr || out == nullptr) { return NXG_ERROR_INVALID_ARGUMENT; }
    *out = nullptr;
    try {
        std::string text(source);
        std::vector<float> frequencies;
        if ((flags & NXG_EXPRESSION_CLASSIC) != 0u) {
            text = nxg::classic_rewrite(nxg::classic_strip(text), frequencies);
        }
        nxg::Parser parser(nxg::lex(nxg::normalise(text)), expression_name ? expression_name : "",
                           object_type ? object_type : "");
        const nxg::Program program = parser.run();
        auto *handle = new (std::nothrow) nxg_expression;
        if (handle == nullptr) { return NXG_ERROR_INVALID_ARGUMENT; }
        static_cast<Expression &>(*handle) = nxg::to_float_program(program, std::move(frequencies));
        *out = handle;
        nxg::copy_message("", message, message_capacity);
        return NXG_ERROR_NONE;
    } catch (const nxg::CompileError &e) {
        nxg::copy_message(e.text, message, message_capacity);
    } catch (const std::exception &e) {
        nxg::copy_message(e.what(), message, message_capacity);
    }
    return NXG_ERROR_EXPRESSION_SYNTAX;
}

void nxg_expression_destroy(nxg_expression *expression) { delete expression; }

uint32_t nxg_expression_get_info(const nxg_expression *e, nxg_expression_info *info) {
    if (e == nullptr || info == nullptr) { return NXG_ERROR_INVALID_ARGUMENT; }
    std::memset(info, 0, sizeof *info);
    info->instruction_count = static_cast<uint32_t>(e->instructions.size());
    info->operand_count = static_cast<uint32_t>(e->operands.size());
    info->input_count = static_cast<uint32_t>(e->inputs.size());
    info->ramp_count = static_cast<uint32_t>(e->ramps.size());
    info->ramp_point_count = static_cast<uint32_t>(e->ramp_points.size());
    info->result = e->result;
    info->expression_seed = e->expression_seed;
    info->random_call_count = e->random_call_count;
    info->pref_noise_count = static_cast<uint32_t>(e->pref_noise.size());
    for (size_t i = 0; i < e->pref_noise.size() && i < NXG_EXPRESSION_MAX_INPUTS; ++i) {
        info->pref_noise_frequencies[i] = e->pref_noise[i];
    }
    return NXG_ERROR_NONE;
}

uint32_t nxg_expression_get_instruction(const nxg_expression *e, uint32_t index,
                                        nxg_expression_instruction *instruction) {
    if (e == nullptr || instruction == nullptr || index >= e->instructions.size()) {
        return NXG_ERROR_INVALID_ARGUMENT;
    }
    const nxg::ExprInstruction &in = e->instructions[index];
    instruction->op = in.op;
    instruction->operand_offset = in.operand_offset;
    instruction->operand_count = in.operand_count;
    instruction->auxiliary = in.auxiliary;
    instruction->immediate = in.immediate;
    return NXG_ERROR_NONE;
}

uint32_t nxg_expression_get_operand(const nxg_expression *e, uint32_t index, uint32_t *operand) {
    if (e == nullptr || operand == nullptr || index >= e->operands.size()) { return NXG_ERROR_INVALID_ARGUMENT; }
    *operand = e->operands[index];
    return NXG_ERROR_NONE;
}

uint32_t nxg_expression_get_ramp_point(const nxg_expression *e, uint32_t index, nxg_expression_ramp_point *point) {
    if (e == nullptr || point == nullptr || index >= e->ramp_points.size()) { return NXG_ERROR_INVALID_ARGUMENT; }
    point->position = e->ramp_points[index].position;
    point->value = e->ramp_points[index].value;
    point->interpolation = e->ramp_points[index].interpolation;
    return NXG_ERROR_NONE;
}

const char *nxg_expression_input_name(const nxg_expression *e, uint32_t index) {
    if (e == nullptr || index >= e->inputs.size()) { return nullptr; }
    return e->inputs[index].c_str();
}

uint32_t nxg_xgen_string_seed(const char *text) { return nxg::string_seed(text ? std::string(text) : std::string()); }

} // extern "C"
