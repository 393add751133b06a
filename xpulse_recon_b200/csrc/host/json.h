// json.h -- minimal JSON reader / writer for the XPRecon parameter files.
//
// Accepts standard JSON plus what the reference's documented examples use:
// // and /* */ comments and trailing commas (README.md:50-85).
#pragma once

#include <cstdint>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

namespace xpr {
namespace json {

struct Value {
    enum Type { Null, Bool, Number, String, Array, Object };
    Type type = Null;
    bool b = false;
    double num = 0.0;
    std::string str;
    std::vector<Value> arr;
    std::vector<std::pair<std::string, Value>> obj;

    const Value *get(const std::string &key) const;
    bool is_object() const { return type == Object; }
};

struct ParseError : std::runtime_error {
    using std::runtime_error::runtime_error;
};

Value parse(const std::string &text);
std::string quote(const std::string &s);

}  // namespace json
}  // namespace xpr
