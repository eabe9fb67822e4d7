// ron.cpp -- see ron.h.
#include "ron.h"

#include <cerrno>

#include <cctype>
#include <cstdlib>
#include <sstream>

namespace necsim {
namespace ron {

namespace {

struct Reader {
    const std::string &s;
    size_t i = 0;
    size_t line = 1;

    [[noreturn]] void error(const std::string &m) const { throw ParseError{m, line}; }

    void skip() {
        for (;;) {
            while (i < s.size() && std::isspace((unsigned char)s[i])) {
                if (s[i] == '\n') ++line;
                ++i;
            }
            if (i + 1 < s.size() && s[i] == '/' && s[i + 1] == '/') {
                while (i < s.size() && s[i] != '\n') ++i;
                continue;
            }
            if (i + 1 < s.size() && s[i] == '/' && s[i + 1] == '*') {
                // block comments nest in RON
                int depth = 0;
                do {
                    if (i + 1 >= s.size()) error("unterminated block comment");
                    if (s[i] == '/' && s[i + 1] == '*') {
                        ++depth;
                        i += 2;
                    } else if (s[i] == '*' && s[i + 1] == '/') {
                        --depth;
                        i += 2;
                    } else {
                        if (s[i] == '\n') ++line;
                        ++i;
                    }
                } while (depth > 0);
                continue;
            }
            return;
        }
    }

    bool peek(char c) {
        skip();
        return i < s.size() && s[i] == c;
    }

    void expect(char c) {
        if (!peek(c)) error(std::string("expected '") + c + "'");
        ++i;
    }

    std::string ident() {
        skip();
        size_t b = i;
        while (i < s.size() && (std::isalnum((unsigned char)s[i]) || s[i] == '_')) ++i;
        if (b == i) error("expected an identifier");
        return s.substr(b, i - b);
    }

    Value value() {
        skip();
        if (i >= s.size()) error("unexpected end of input");
        const char c = s[i];
        Value v;
        if (c == '"') {
            ++i;
            v.kind = Value::String;
            while (i < s.size() && s[i] != '"') {
                if (s[i] == '\\' && i + 1 < s.size()) {
                    const char e = s[i + 1];
                    v.text += (e == 'n') ? '\n' : (e == 't') ? '\t' : e;
                    i += 2;
                } else {
                    if (s[i] == '\n') ++line;
                    v.text += s[i++];
                }
            }
            if (i >= s.size()) error("unterminated string");
            ++i;
            return v;
        }
        if (c == '-' || c == '+' || c == '.' || std::isdigit((unsigned char)c)) {
            size_t b = i;
            if (s[i] == '-' || s[i] == '+') ++i;
            while (i < s.size() && (std::isalnum((unsigned char)s[i]) || s[i] == '.' || s[i] == '_' ||
                                    ((s[i] == '-' || s[i] == '+') && (s[i - 1] == 'e' || s[i - 1] == 'E'))))
                ++i;
            v.kind = Value::Number;
            for (size_t k = b; k < i; ++k)
                if (s[k] != '_') v.text += s[k];
            return v;
        }
        if (c == '[') {
            ++i;
            v.kind = Value::List;
            while (!peek(']')) {
                v.items.push_back(value());
                if (!peek(',')) break;
                ++i;
            }
            expect(']');
            return v;
        }
        if (c == '(' || std::isalpha((unsigned char)c) || c == '_') {
            if (c != '(') {
                v.text = ident();
                if (v.text == "true" || v.text == "false") {
                    v.kind = Value::Bool;
                    v.boolean = v.text == "true";
                    return v;
                }
                v.kind = Value::Ident;
                if (!peek('(')) return v;
            }
            // (named) struct or tuple
            expect('(');
            v.kind = Value::Struct;
            while (!peek(')')) {
                // `name: value` or a positional value
                size_t save = i, save_line = line;
                bool named = false;
                skip();
                if (i < s.size() && (std::isalpha((unsigned char)s[i]) || s[i] == '_')) {
                    std::string name = ident();
                    if (peek(':')) {
                        ++i;
                        v.fields.emplace_back(name, value());
                        named = true;
                    }
                }
                if (!named) {
                    i = save;
                    line = save_line;
                    v.items.push_back(value());
                }
                if (!peek(',')) break;
                ++i;
            }
            expect(')');
            return v;
        }
        error(std::string("unexpected character '") + c + "'");
    }
};

}  // namespace

double Value::as_f64() const {
    if (kind != Number) throw ParseError{"expected a number, found " + text, 0};
    char *end = nullptr;
    const double d = std::strtod(text.c_str(), &end);
    if (!end || *end) throw ParseError{"malformed number " + text, 0};
    return d;
}

uint64_t Value::as_u64() const {
    if (kind != Number) throw ParseError{"expected an integer, found " + text, 0};
    char *end = nullptr;
    const unsigned long long u = std::strtoull(text.c_str(), &end, 10);
    if (!end || *end || text.empty() || text[0] == '-') throw ParseError{"malformed integer " + text, 0};
    return u;
}

int64_t Value::as_i64() const {
    if (kind != Number) throw ParseError{"expected an integer, found " + text, 0};
    char *end = nullptr;
    errno = 0;
    const long long v = std::strtoll(text.c_str(), &end, 10);
    if (!end || *end || text.empty() || errno == ERANGE) throw ParseError{"malformed i64 " + text, 0};
    return v;
}

const Value *Value::field(const std::string &name) const {
    for (const auto &f : fields)
        if (f.first == name) return &f.second;
    return nullptr;
}

Value parse(const std::string &src) {
    Reader r{src};
    Value v = r.value();
    r.skip();
    if (r.i != src.size()) r.error("trailing characters after the value");
    return v;
}

std::string to_string(const Value &v, int indent) {
    const std::string pad(indent + 4, ' '), end_pad(indent, ' ');
    switch (v.kind) {
    case Value::Number:
        return v.text;
    case Value::String: {
        std::string o = "\"";
        for (char c : v.text) {
            if (c == '"' || c == '\\') o += '\\';
            o += c;
        }
        return o + "\"";
    }
    case Value::Bool:
        return v.boolean ? "true" : "false";
    case Value::Ident:
        return v.text;
    case Value::List: {
        if (v.items.empty()) return "[]";
        std::string o = "[\n";
        for (const auto &x : v.items) o += pad + to_string(x, indent + 4) + ",\n";
        return o + end_pad + "]";
    }
    case Value::Struct: {
        std::string o = v.text + "(";
        if (v.fields.empty() && v.items.empty()) return o + ")";
        o += "\n";
        for (const auto &f : v.fields) o += pad + f.first + ": " + to_string(f.second, indent + 4) + ",\n";
        for (const auto &x : v.items) o += pad + to_string(x, indent + 4) + ",\n";
        return o + end_pad + ")";
    }
    }
    return "";
}

}  // namespace ron
}  // namespace necsim
