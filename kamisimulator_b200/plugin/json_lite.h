// json_lite.h -- a small reader for flat JSON settings objects: string keys mapping to numbers,
// booleans, strings or arrays of numbers (the shape of KamiSimulator's solver settings files).
#pragma once
#include <map>
#include <string>
#include <vector>

namespace kami {

struct JsonValue {
    enum Kind { Number, Bool, String, Array, Other } kind = Other;
    double number = 0.0;
    bool boolean = false;
    std::string text;
    std::vector<double> array;
};

// Parses a JSON object; throws std::runtime_error on malformed input.
std::map<std::string, JsonValue> parse_json_object(const std::string& text);

}  // namespace kami
