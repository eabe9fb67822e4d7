// ron.h -- a reader for the subset of RON (Rusty Object Notation) that
// rustcoalescence's configuration files use: numbers, strings, booleans,
// identifiers / unit enum variants, named and anonymous structs and tuples
// `Name(a: 1, b: (2, 3))`, lists `[...]`, `//` and `/* */` comments and
// trailing commas.
#pragma once

#include <cstdint>
#include <map>
#include <memory>
#include <string>
#include <vector>

namespace necsim {
namespace ron {

struct Value {
    enum Kind { Number, String, Bool, Ident, Struct, List } kind = Ident;
    std::string text;                  // number literal, string contents or identifier / struct name
    bool boolean = false;
    std::vector<std::pair<std::string, Value>> fields;  // Struct: named fields (in order)
    std::vector<Value> items;          // Struct: positional members; List: elements

    bool is_number() const { return kind == Number; }
    double as_f64() const;
    uint64_t as_u64() const;
    int64_t as_i64() const;
    // Struct field by name (nullptr when absent)
    const Value *field(const std::string &name) const;
    // `Name` or `Name(...)`: the variant name of an enum value
    const std::string &variant() const { return text; }
};

struct ParseError {
    std::string msg;
    size_t line;
};

// Parses one RON value (the whole document); throws ParseError.
Value parse(const std::string &src);

// Writes a value back as RON (used for resume configurations).
std::string to_string(const Value &v, int indent = 0);

}  // namespace ron
}  // namespace necsim
