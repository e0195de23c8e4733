// expression.cpp -- host compiler for XGen scalar expressions.
//
// Produces the SSA program that the device evaluator (classic.cu) runs for
// every root.  The language, the compiled program (instruction numbering,
// operand order, emission order) and the error texts are the reference
// compiler's; the code is a reader that rewrites comments and line breaks on
// the fly, a one-pass scanner and a precedence-climbing parser.  Behaviour
// followed:
//   source rewriting (comments, "\n", line joining)  src/xgen_expression.cpp:50-118
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

#include <algorithm>
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

// --------------------------------------------------------------- reading
//
// The language is defined on a rewritten form of the source: the two
// characters "\n" stand for a newline, '#' comments run to the end of their
// line and become a statement break (';'), and every remaining newline joins
// the two lines (a space) when the text before it ends, or the text after it
// starts, with an operator, and separates statements (';') otherwise.  Error
// offsets count bytes of that rewritten form.  Reader produces it one
// character at a time, so the scanner below never sees a rewritten copy of
// the source; it also reports, for each character it hands out, where the
// character sits in the source (numbers are parsed in place there).
class Reader {
public:
    explicit Reader(const std::string &source) : src_(source) {
        if (src_.size() > kMaxSourceBytes) { fail("XGen scalar expression source byte limit exceeded"); }
        if (src_.find('\0') != std::string::npos) { fail("XGen scalar expression contains a NUL byte"); }
    }

    // The character `ahead` positions on (0 = the next one), or -1 past the end.
    int peek(size_t ahead = 0) {
        while (pending_.size() <= ahead) {
            if (!produce()) { return -1; }
        }
        return static_cast<unsigned char>(pending_[ahead].c);
    }
    int next() {
        const int c = peek();
        if (c >= 0) {
            pending_.erase(pending_.begin());
            ++offset_;
        }
        return c;
    }
    // Rewritten-form offset of the next character.
    size_t offset() const { return offset_; }
    // Source position of the next character; the source itself.
    size_t source_position() {
        peek();
        return pending_.empty() ? src_.size() : pending_.front().at;
    }
    const std::string &source() const { return src_; }

private:
    struct Pending {
        char c;
        size_t at;
    };

    // Operators that carry an expression over a line break.
    static bool joins(char c) { return std::strchr("+-*/<>=!&|?:,(", c) != nullptr; }
    static bool line_end(char c) { return c == '\n' || c == '\r'; }

    // The source character at `pos`, with the "\n" escape read as a newline;
    // `width` is how many source bytes it spans.
    char logical(size_t pos, size_t &width) const {
        if (src_[pos] == '\\' && pos + 1 < src_.size() && src_[pos + 1] == 'n') {
            width = 2;
            return '\n';
        }
        width = 1;
        return src_[pos];
    }

    // Whether the first character after a line break (blanks and further
    // line breaks skipped) starts with a joining operator or ')'.  A comment
    // there counts as a statement break.
    bool next_line_joins(size_t pos) const {
        while (pos < src_.size()) {
            size_t width = 0;
            const char c = logical(pos, width);
            if (c != ' ' && c != '\t' && !line_end(c)) { return c != '#' && (joins(c) || c == ')'); }
            pos += width;
        }
        return false;
    }

    void emit(char c, size_t at) {
        pending_.push_back(Pending{c, at});
        if (c != ' ' && c != '\t') { last_solid_ = c; }
    }

    // Appends the next rewritten character(s); false at the end of the source.
    bool produce() {
        while (pos_ < src_.size()) {
            size_t width = 0;
            const size_t at = pos_;
            const char c = logical(pos_, width);
            pos_ += width;
            if (c == '#') {  // skip to the line end, which the comment consumes
                while (pos_ < src_.size()) {
                    const char d = logical(pos_, width);
                    pos_ += width;
                    if (line_end(d)) {
                        emit(';', at);
                        return true;
                    }
                }
                return false;
            }
            if (line_end(c)) {
                emit((last_solid_ != 0 && joins(last_solid_)) || next_line_joins(pos_) ? ' ' : ';', at);
                return true;
            }
            emit(c, at);
            return true;
        }
        return false;
    }

    const std::string &src_;
    size_t pos_ = 0;
    size_t offset_ = 0;
    char last_solid_ = 0;  // the last character handed on other than a blank
    std::vector<Pending> pending_;
};

// -------------------------------------------------------------- scanning

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

bool ident_start(int c) { return (c >= 'a' && c <= 'z') || (c >= 'A' && c <= 'Z') || c == '_'; }
bool ident_part(int c) { return ident_start(c) || (c >= '0' && c <= '9'); }
bool is_digit(int c) { return c >= '0' && c <= '9'; }

// Punctuation: a character, optionally followed by a second one that makes a
// different token (`pair`), else `single` -- or, where the character has no
// meaning alone, the error text `alone`.
struct Punct {
    char first, second;
    Tok pair, single;
    const char *alone;
};
constexpr Punct kPunctuation[] = {
    {';', 0, Tok::End, Tok::Semicolon, nullptr}, {',', 0, Tok::End, Tok::Comma, nullptr},
    {'(', 0, Tok::End, Tok::LParen, nullptr},    {')', 0, Tok::End, Tok::RParen, nullptr},
    {'?', 0, Tok::End, Tok::Question, nullptr},  {':', 0, Tok::End, Tok::Colon, nullptr},
    {'+', 0, Tok::End, Tok::Plus, nullptr},      {'*', 0, Tok::End, Tok::Star, nullptr},
    {'/', 0, Tok::End, Tok::Slash, nullptr},     {'-', '>', Tok::Arrow, Tok::Minus, nullptr},
    {'=', '=', Tok::Equal, Tok::Assign, nullptr}, {'!', '=', Tok::NotEqual, Tok::Bang, nullptr},
    {'<', '=', Tok::LessEqual, Tok::Less, nullptr}, {'>', '=', Tok::GreaterEqual, Tok::Greater, nullptr},
    {'&', '&', Tok::And, Tok::End, "single '&' is unsupported; use '&&'"},
    {'|', '|', Tok::Or, Tok::End, "single '|' is unsupported; use '||'"},
};

// The whole token list of a source (the parser looks two tokens ahead).
std::vector<Token> scan(const std::string &source) {
    Reader in(source);
    std::vector<Token> tokens;
    const auto add = [&tokens](Token t) {
        if (tokens.size() >= kMaxTokens) { fail("XGen scalar expression token limit exceeded"); }
        tokens.push_back(std::move(t));
    };
    for (;;) {
        const int c = in.peek();
        const size_t at = in.offset();
        if (c < 0) { break; }
        if (c == ' ' || c == '\t' || c == '\f' || c == '\v') {
            in.next();
            continue;
        }
        Token t;
        t.offset = at;
        if (is_digit(c) || (c == '.' && is_digit(in.peek(1)))) {
            // strtod in place: a literal never spans a rewritten character.
            const char *first = in.source().c_str() + in.source_position();
            char *last = nullptr;
            t.number = std::strtod(first, &last);
            const size_t length = static_cast<size_t>(last - first);
            if (length == 0 || !std::isfinite(t.number)) { syntax(at, "invalid or non-finite numeric literal"); }
            for (size_t k = 0; k < length; ++k) { in.next(); }
            t.kind = Tok::Number;
        } else if (c == '$' || ident_start(c)) {
            t.kind = c == '$' ? Tok::Variable : Tok::Identifier;
            if (c == '$') {
                in.next();
                if (!ident_start(in.peek())) { syntax(at, "expected a variable name after '$'"); }
            }
            while (ident_part(in.peek())) { t.text.push_back(static_cast<char>(in.next())); }
        } else if (c == '\'' || c == '"') {
            in.next();
            for (int d = in.next();; d = in.next()) {
                if (d < 0) { syntax(at, "unterminated string literal"); }
                if (d == c) { break; }
                if (d == '\\' && in.peek() >= 0) { d = in.next(); }
                t.text.push_back(static_cast<char>(d));
            }
            t.kind = Tok::String;
        } else {
            const Punct *p = nullptr;
            for (const Punct &q : kPunctuation) {
                if (q.first == c) { p = &q; }
            }
            if (p == nullptr) { syntax(at, "unsupported character"); }
            in.next();
            if (p->second != 0 && in.peek() == p->second) {
                in.next();
                t.kind = p->pair;
            } else if (p->alone != nullptr) {
                syntax(at, p->alone);
            } else {
                t.kind = p->single;
            }
        }
        add(std::move(t));
    }
    Token end;
    end.offset = in.offset();
    add(std::move(end));
    return tokens;
}

// --------------------------------------------------------------- parsing
//
// Precedence climbing over a binding-power table.  Binary operators bind
// tighter the higher their power and associate to the left; the conditional
// a ? b : c binds loosest and associates to the right; prefix + - ! apply to
// an operand, which is a primary value followed by any ->method(...) calls.
// Operands are emitted before the instruction that uses them, so every value
// is an SSA index into the instruction list; locals alias earlier values.

struct Binary {
    Tok token;
    int power;
    ExprOp op;
};
constexpr Binary kBinary[] = {
    {Tok::Or, 1, kOpLogicalOr},        {Tok::And, 2, kOpLogicalAnd},
    {Tok::Equal, 3, kOpEqual},          {Tok::NotEqual, 3, kOpNotEqual},
    {Tok::Less, 4, kOpLess},            {Tok::LessEqual, 4, kOpLessEqual},
    {Tok::Greater, 4, kOpGreater},      {Tok::GreaterEqual, 4, kOpGreaterEqual},
    {Tok::Plus, 5, kOpAdd},             {Tok::Minus, 5, kOpSubtract},
    {Tok::Star, 6, kOpMultiply},        {Tok::Slash, 6, kOpDivide},
};

const Binary *binary_of(Tok t) {
    for (const Binary &b : kBinary) {
        if (b.token == t) { return &b; }
    }
    return nullptr;
}

// Intrinsics by name: the op and the argument count (-1: any count from 1).
struct Intrinsic {
    const char *name;
    ExprOp op;
    int arity;
};
constexpr Intrinsic kIntrinsics[] = {
    {"hash", kOpHash, -1},    {"min", kOpMinimum, 2},      {"max", kOpMaximum, 2},
    {"clamp", kOpClamp, 3},   {"fit", kOpFit, 5},          {"gamma", kOpGamma, 2},
    {"contrast", kOpContrast, 2}, {"smoothstep", kOpSmoothstep, 3},
};

class Compiler {
public:
    Compiler(std::vector<Token> tokens, const std::string &name, const std::string &type)
        : tokens_(std::move(tokens)) {
        program_.expression_seed = string_seed(name + type);
    }

    // statements := statement (';' statement)*, where a statement is
    // `name = value` (with or without '$') or a value; the last statement's
    // value is the result.
    Program compile() {
        bool any = false;
        for (;;) {
            while (at(Tok::Semicolon)) { ++cursor_; }
            if (at(Tok::End)) { break; }
            const bool assignment = (at(Tok::Variable) || at(Tok::Identifier)) && ahead(1).kind == Tok::Assign;
            std::string target;
            if (assignment) {
                target = ahead(0).text;
                cursor_ += 2;
            }
            const uint32_t value = value_of(0);
            if (assignment) {
                if (!locals_.count(target) && locals_.size() >= kMaxLocals) {
                    fail("XGen scalar expression local limit exceeded");
                }
                locals_[target] = value;
            }
            program_.result = value;
            any = true;
            if (!at(Tok::Semicolon) && !at(Tok::End)) { syntax(ahead(0).offset, "expected ';' after expression"); }
        }
        if (!any) { syntax(0, "expression is empty"); }
        return std::move(program_);
    }

private:
    const Token &ahead(size_t k) const { return tokens_[std::min(cursor_ + k, tokens_.size() - 1)]; }
    bool at(Tok t) const { return ahead(0).kind == t; }
    bool eat(Tok t) {
        if (!at(t)) { return false; }
        ++cursor_;
        return true;
    }
    void need(Tok t, const char *message) {
        if (!eat(t)) { syntax(ahead(0).offset, message); }
    }

    uint32_t emit(ExprOp op, const std::vector<uint32_t> &operands = {}, double immediate = 0.0,
                  uint32_t auxiliary = 0) {
        if (program_.instructions.size() >= kMaxInstructions) {
            fail("XGen scalar expression instruction limit exceeded");
        }
        if (operands.size() > std::numeric_limits<uint16_t>::max()) {
            fail("XGen scalar expression operand limit exceeded");
        }
        const size_t first = program_.operands.size();
        if (first > std::numeric_limits<uint32_t>::max()) { fail("XGen scalar expression operand storage exceeded"); }
        program_.operands.insert(program_.operands.end(), operands.begin(), operands.end());
        program_.instructions.push_back(Instruction{static_cast<uint8_t>(op), static_cast<uint32_t>(first),
                                                    static_cast<uint16_t>(operands.size()), auxiliary, immediate});
        return static_cast<uint32_t>(program_.instructions.size() - 1);
    }

    // A value whose binary operators all bind tighter than `floor`; at floor
    // 0 a trailing conditional is taken as well.
    uint32_t value_of(int floor) {
        uint32_t left = operand();
        for (;;) {
            if (floor == 0 && eat(Tok::Question)) {
                const uint32_t yes = value_of(0);
                need(Tok::Colon, "expected ':' in conditional expression");
                const uint32_t no = value_of(0);
                left = emit(kOpSelect, {left, yes, no});
                continue;
            }
            const Binary *b = binary_of(ahead(0).kind);
            if (b == nullptr || b->power <= floor) { return left; }
            ++cursor_;
            const uint32_t right = value_of(b->power);
            left = emit(b->op, {left, right});
        }
    }

    // Prefix operators, then a primary value and its method calls.
    uint32_t operand() {
        if (eat(Tok::Plus)) { return operand(); }
        if (eat(Tok::Minus)) { return emit(kOpNegate, {operand()}); }
        if (eat(Tok::Bang)) { return emit(kOpLogicalNot, {operand()}); }
        uint32_t v = primary();
        while (eat(Tok::Arrow)) {
            if (!at(Tok::Identifier)) { syntax(ahead(0).offset, "expected a method name after '->'"); }
            const Token name = tokens_[cursor_++];
            need(Tok::LParen, "expected '(' after expression method name");
            std::vector<uint32_t> arguments{v};
            arguments_until_paren(arguments, "expected ')' after expression method arguments");
            v = intrinsic(name, arguments);
        }
        return v;
    }

    // Comma-separated values up to ')', appended to `out` (the '(' is taken).
    void arguments_until_paren(std::vector<uint32_t> &out, const char *unclosed) {
        if (eat(Tok::RParen)) { return; }
        do {
            out.push_back(value_of(0));
        } while (eat(Tok::Comma));
        need(Tok::RParen, unclosed);
    }

    uint32_t primary() {
        const Token &t = ahead(0);
        switch (t.kind) {
            case Tok::Number:
                ++cursor_;
                return emit(kOpConstant, {}, t.number);
            case Tok::Variable: {
                ++cursor_;
                const auto local = locals_.find(t.text);
                if (local != locals_.end()) { return local->second; }
                const auto known = std::find(program_.inputs.begin(), program_.inputs.end(), t.text);
                const uint32_t index = static_cast<uint32_t>(known - program_.inputs.begin());
                if (known == program_.inputs.end()) { program_.inputs.push_back(t.text); }
                return emit(kOpInput, {}, 0.0, index);
            }
            case Tok::LParen: {
                ++cursor_;
                const uint32_t v = value_of(0);
                need(Tok::RParen, "expected ')'");
                return v;
            }
            case Tok::String:
                syntax(t.offset, "string values require an explicit PTEX binding such as map()");
            case Tok::Identifier:
                break;
            default:
                syntax(t.offset, "expected a scalar value");
        }
        const Token name = tokens_[cursor_++];
        if (name.text == "true" || name.text == "false") { return emit(kOpConstant, {}, name.text == "true"); }
        if (!eat(Tok::LParen)) {
            const auto local = locals_.find(name.text);
            if (local == locals_.end()) { syntax(name.offset, "bare identifier is unsupported: " + name.text); }
            return local->second;
        }
        if (name.text == "rampUI") { return ramp(name.offset); }
        std::vector<uint32_t> arguments;
        arguments_until_paren(arguments, "expected ')' after function arguments");
        return intrinsic(name, arguments);
    }

    uint32_t intrinsic(const Token &name, const std::vector<uint32_t> &arguments) {
        const std::string &f = name.text;
        if (f == "rand") {
            if (arguments.size() > 3) { syntax(name.offset, "rand expects zero to three arguments"); }
            // Each call site draws its own seed from (expression seed, call number).
            const double site[2] = {static_cast<double>(program_.expression_seed),
                                    static_cast<double>(program_.random_call_count++)};
            return emit(kOpRandom, arguments, seexpr_hash(site, 2));
        }
        if (f == "map") {
            syntax(name.offset, "map requires an explicit PTEX binding and is not a scalar intrinsic");
        }
        for (const Intrinsic &in : kIntrinsics) {
            if (f != in.name) { continue; }
            if (in.arity < 0 && arguments.empty()) { syntax(name.offset, f + " expects at least one argument"); }
            if (in.arity >= 0 && arguments.size() != static_cast<size_t>(in.arity)) {
                syntax(name.offset, f + " expects " + std::to_string(in.arity) + " argument(s)");
            }
            return emit(in.op, arguments);
        }
        syntax(name.offset, "unsupported function: " + f);
    }

    // One signed numeric field of a rampUI point.
    double ramp_field(const char *what) {
        const double sign = eat(Tok::Plus) ? 1.0 : (eat(Tok::Minus) ? -1.0 : 1.0);
        if (!at(Tok::Number)) { syntax(ahead(0).offset, std::string("expected a numeric ramp ") + what); }
        return sign * tokens_[cursor_++].number;
    }

    // rampUI(position, value, interpolation : ...) after its '('.  Points are
    // checked as they are read; errors point at the rampUI name.
    uint32_t ramp(size_t where) {
        const size_t first = program_.ramp_points.size();
        do {
            RampPoint point{};
            point.position = ramp_field("position");
            need(Tok::Comma, "expected ',' after ramp position");
            point.value = ramp_field("value");
            need(Tok::Comma, "expected ',' after ramp value");
            const double kind = ramp_field("interpolation");
            if (kind < 0.0 || kind > 3.0 || kind != std::floor(kind)) {
                syntax(where, "ramp interpolation must be an integer in [0, 3]");
            }
            if (!(point.position >= 0.0 && point.position <= 1.0)) {
                syntax(where, "ramp positions must be in [0, 1]");
            }
            if (program_.ramp_points.size() >= kMaxRampPoints) { fail("XGen scalar expression ramp point limit exceeded"); }
            if (program_.ramp_points.size() > first && !(point.position > program_.ramp_points.back().position)) {
                syntax(where, "ramp positions must be strictly increasing");
            }
            point.interpolation = static_cast<uint8_t>(kind);
            program_.ramp_points.push_back(point);
        } while (eat(Tok::Colon));
        need(Tok::RParen, "expected ')' after rampUI points");
        const size_t count = program_.ramp_points.size() - first;
        if (count == 0 || count > std::numeric_limits<uint16_t>::max() ||
            first > std::numeric_limits<uint32_t>::max()) {
            syntax(where, "ramp point storage limit exceeded");
        }
        program_.ramps.push_back(ExprRamp{static_cast<uint32_t>(first), static_cast<uint32_t>(count)});
        return emit(kOpRamp, {}, 0.0, static_cast<uint32_t>(program_.ramps.size() - 1));
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
        nxg::Compiler compiler(nxg::scan(text), expression_name ? expression_name : "",
                               object_type ? object_type : "");
        const nxg::Program program = compiler.compile();
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
