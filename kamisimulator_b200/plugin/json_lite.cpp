// json_lite.cpp -- see json_lite.h.
#include "json_lite.h"

#include <cctype>
#include <cstdlib>
#include <stdexcept>

namespace kami {
namespace {

struct Reader {
    const std::string& s;
    size_t i = 0;
    explicit Reader(const std::string& t) : s(t) {}
    void ws() {
        while (i < s.size() && std::isspace((unsigned char)s[i])) i++;
    }
    [[noreturn]] void error(const char* what) {
        throw std::runtime_error(std::string("settings JSON: ") + what + " at offset " + std::to_string(i));
    }
    char peek() {
        ws();
        if (i >= s.size()) error("unexpected end");
        return s[i];
    }
    void expect(char c) {
        if (peek() != c) error((std::string("expected '") + c + "'").c_str());
        i++;
    }
    std::string str() {
        expect('"');
        std::string out;
        while (i < s.size() && s[i] != '"') {
            if (s[i] == '\\' && i + 1 < s.size()) i++;
            out += s[i++];
        }
        if (i >= s.size()) error("unterminated string");
        i++;
        return out;
    }
    double num() {
        ws();
        const char* b = s.c_str() + i;
        char* e = nullptr;
        double v = std::strtod(b, &e);
        if (e == b) error("expected a number");
        i += (size_t)(e - b);
        return v;
    }
    void skip_value() {  // nested objects are skipped
        char c = peek();
        if (c == '{' || c == '[') {
            int depth = 0;
            do {
                if (s[i] == '"') {
                    str();
                    continue;
                }
                if (s[i] == '{' || s[i] == '[') depth++;
                if (s[i] == '}' || s[i] == ']') depth--;
                i++;
            } while (depth > 0 && i < s.size());
        } else if (c == '"') {
            str();
        } else {
            while (i < s.size() && s[i] != ',' && s[i] != '}') i++;
        }
    }
    JsonValue value() {
        JsonValue v;
        char c = peek();
        if (c == '"') {
            v.kind = JsonValue::String;
            v.text = str();
        } else if (c == 't' || c == 'f') {
            v.kind = JsonValue::Bool;
            v.boolean = s.compare(i, 4, "true") == 0;
            i += v.boolean ? 4 : 5;
        } else if (c == '[') {
            size_t save = i;
            i++;
            v.kind = JsonValue::Array;
            if (peek() == ']') {
                i++;
                return v;
            }
            while (true) {
                char d = peek();
                if (!(d == '-' || d == '+' || d == '.' || std::isdigit((unsigned char)d))) {
                    i = save;
                    skip_value();
                    v.kind = JsonValue::Other;
                    return v;
                }
                v.array.push_back(num());
                if (peek() == ',') {
                    i++;
                    continue;
                }
                expect(']');
                break;
            }
        } else if (c == '{' || c == 'n') {
            skip_value();
            v.kind = JsonValue::Other;
        } else {
            v.kind = JsonValue::Number;
            v.number = num();
        }
        return v;
    }
};

}  // namespace

std::map<std::string, JsonValue> parse_json_object(const std::string& text) {
    Reader r(text);
    std::map<std::string, JsonValue> out;
    r.expect('{');
    if (r.peek() == '}') return out;
    while (true) {
        std::string key = r.str();
        r.expect(':');
        out[key] = r.value();
        char c = r.peek();
        r.i++;
        if (c == '}') break;
        if (c != ',') r.error("expected ',' or '}'");
    }
    return out;
}

}  // namespace kami
