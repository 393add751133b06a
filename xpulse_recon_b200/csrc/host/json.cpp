// json.cpp -- see json.h
#include "json.h"

#include <cstdlib>
#include <cstring>

namespace xpr {
namespace json {

const Value *Value::get(const std::string &key) const
{
    if (type != Object) return nullptr;
    for (const auto &kv : obj)
        if (kv.first == key) return &kv.second;
    return nullptr;
}

namespace {

struct Parser {
    const std::string &t;
    size_t i = 0;

    explicit Parser(const std::string &text) : t(text) {}

    [[noreturn]] void fail(const char *what) const
    {
        size_t line = 1, col = 1;
        for (size_t k = 0; k < i && k < t.size(); ++k) {
            if (t[k] == '\n') { ++line; col = 1; } else { ++col; }
        }
        throw ParseError(std::string("JSON: ") + what + " at line " + std::to_string(line) + ", column " +
                         std::to_string(col));
    }

    void skip()
    {
        for (;;) {
            while (i < t.size() && (t[i] == ' ' || t[i] == '\t' || t[i] == '\n' || t[i] == '\r')) ++i;
            if (i + 1 < t.size() && t[i] == '/' && t[i + 1] == '/') {
                while (i < t.size() && t[i] != '\n') ++i;
                continue;
            }
            if (i + 1 < t.size() && t[i] == '/' && t[i + 1] == '*') {
                size_t e = t.find("*/", i + 2);
                if (e == std::string::npos) fail("unterminated comment");
                i = e + 2;
                continue;
            }
            break;
        }
    }

    bool eat(char c)
    {
        skip();
        if (i < t.size() && t[i] == c) { ++i; return true; }
        return false;
    }

    std::string string_lit()
    {
        if (!eat('"')) fail("expected a string");
        std::string out;
        while (i < t.size() && t[i] != '"') {
            char c = t[i++];
            if (c != '\\') { out.push_back(c); continue; }
            if (i >= t.size()) fail("bad escape");
            char e = t[i++];
            switch (e) {
                case '"': out.push_back('"'); break;
                case '\\': out.push_back('\\'); break;
                case '/': out.push_back('/'); break;
                case 'b': out.push_back('\b'); break;
                case 'f': out.push_back('\f'); break;
                case 'n': out.push_back('\n'); break;
                case 'r': out.push_back('\r'); break;
                case 't': out.push_back('\t'); break;
                case 'u': {
                    if (i + 4 > t.size()) fail("bad \\u escape");
                    unsigned cp = (unsigned)std::strtoul(t.substr(i, 4).c_str(), nullptr, 16);
                    i += 4;
                    if (cp < 0x80) out.push_back((char)cp);
                    else if (cp < 0x800) { out.push_back((char)(0xC0 | (cp >> 6))); out.push_back((char)(0x80 | (cp & 0x3F))); }
                    else { out.push_back((char)(0xE0 | (cp >> 12))); out.push_back((char)(0x80 | ((cp >> 6) & 0x3F))); out.push_back((char)(0x80 | (cp & 0x3F))); }
                    break;
                }
                default: fail("bad escape");
            }
        }
        if (i >= t.size()) fail("unterminated string");
        ++i;
        return out;
    }

    Value value()
    {
        skip();
        if (i >= t.size()) fail("unexpected end of input");
        Value v;
        char c = t[i];
        if (c == '{') {
            ++i;
            v.type = Value::Object;
            if (eat('}')) return v;
            for (;;) {
                skip();
                if (i < t.size() && t[i] == '}') { ++i; break; }  // trailing comma
                std::string k = string_lit();
                if (!eat(':')) fail("expected ':'");
                v.obj.emplace_back(k, value());
                if (eat(',')) continue;
                if (eat('}')) break;
                fail("expected ',' or '}'");
            }
            return v;
        }
        if (c == '[') {
            ++i;
            v.type = Value::Array;
            if (eat(']')) return v;
            for (;;) {
                skip();
                if (i < t.size() && t[i] == ']') { ++i; break; }
                v.arr.push_back(value());
                if (eat(',')) continue;
                if (eat(']')) break;
                fail("expected ',' or ']'");
            }
            return v;
        }
        if (c == '"') {
            v.type = Value::String;
            v.str = string_lit();
            return v;
        }
        if (t.compare(i, 4, "true") == 0) { i += 4; v.type = Value::Bool; v.b = true; return v; }
        if (t.compare(i, 5, "false") == 0) { i += 5; v.type = Value::Bool; v.b = false; return v; }
        if (t.compare(i, 4, "null") == 0) { i += 4; return v; }
        if (c == '-' || c == '+' || c == '.' || (c >= '0' && c <= '9')) {
            const char *start = t.c_str() + i;
            char *end = nullptr;
            v.num = std::strtod(start, &end);
            if (end == start) fail("bad number");
            i += (size_t)(end - start);
            v.type = Value::Number;
            return v;
        }
        fail("unexpected character");
    }
};

}  // namespace

Value parse(const std::string &text)
{
    Parser p(text);
    Value v = p.value();
    p.skip();
    if (p.i != text.size()) p.fail("trailing characters");
    return v;
}

std::string quote(const std::string &s)
{
    std::string o = "\"";
    for (char c : s) {
        switch (c) {
            case '"': o += "\\\""; break;
            case '\\': o += "\\\\"; break;
            case '\n': o += "\\n"; break;
            case '\t': o += "\\t"; break;
            case '\r': o += "\\r"; break;
            default: o.push_back(c);
        }
    }
    return o + "\"";
}

}  // namespace json
}  // namespace xpr
