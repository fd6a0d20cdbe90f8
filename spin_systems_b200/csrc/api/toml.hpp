// A small TOML reader for run configurations: tables, arrays of tables,
// dotted keys, inline tables, arrays (multi-line, trailing commas),
// basic/literal strings, integers, floats, booleans and comments.  It stands
// in for toml++ (not available here) with the same accessors the
// configuration code needs: typed lookups where an integer also reads as a
// float, as toml++'s value<double>() allows.
#pragma once

#include <cstdint>
#include <map>
#include <memory>
#include <optional>
#include <stdexcept>
#include <string>
#include <string_view>
#include <utility>
#include <vector>

namespace spinsim::toml {

struct Value;
using Table = std::vector<std::pair<std::string, Value>>;
using Array = std::vector<Value>;

struct Value {
  enum class Kind { None, String, Integer, Float, Bool, Array, Table };
  Kind kind = Kind::None;
  std::string str;
  std::int64_t integer = 0;
  double number = 0.0;
  bool boolean = false;
  std::shared_ptr<toml::Array> array;
  std::shared_ptr<toml::Table> table;

  [[nodiscard]] bool isTable() const { return kind == Kind::Table; }
  [[nodiscard]] bool isArray() const { return kind == Kind::Array; }
  /// Member of a table, or nullptr.
  [[nodiscard]] const Value* get(std::string_view key) const;
  [[nodiscard]] bool contains(std::string_view key) const { return get(key) != nullptr; }
  [[nodiscard]] std::optional<double> asDouble() const;
  [[nodiscard]] std::optional<std::int64_t> asInt() const;
  [[nodiscard]] std::optional<std::string> asString() const;
  [[nodiscard]] std::optional<bool> asBool() const;
};

struct ParseError : std::runtime_error {
  using std::runtime_error::runtime_error;
};

/// Parses a whole document into its root table; throws ParseError with the
/// line number on malformed input.
[[nodiscard]] Value parse(std::string_view text);

}  // namespace spinsim::toml
