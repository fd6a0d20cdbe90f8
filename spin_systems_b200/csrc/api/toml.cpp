// TOML reader; see toml.hpp.
#include "toml.hpp"

#include <cctype>
#include <cmath>
#include <cstdlib>
#include <format>
#include <limits>

namespace spinsim::toml {

const Value* Value::get(std::string_view key) const {
  if (kind != Kind::Table || !table) return nullptr;
  for (const auto& [k, v] : *table) {
    if (k == key) return &v;
  }
  return nullptr;
}

std::optional<double> Value::asDouble() const {
  if (kind == Kind::Float) return number;
  if (kind == Kind::Integer) return static_cast<double>(integer);
  return std::nullopt;
}

std::optional<std::int64_t> Value::asInt() const {
  if (kind == Kind::Integer) return integer;
  return std::nullopt;
}

std::optional<std::string> Value::asString() const {
  if (kind == Kind::String) return str;
  return std::nullopt;
}

std::optional<bool> Value::asBool() const {
  if (kind == Kind::Bool) return boolean;
  return std::nullopt;
}

namespace {

Value makeTable() {
  Value v;
  v.kind = Value::Kind::Table;
  v.table = std::make_shared<Table>();
  return v;
}

Value makeArray() {
  Value v;
  v.kind = Value::Kind::Array;
  v.array = std::make_shared<Array>();
  return v;
}

class Parser {
 public:
  explicit Parser(std::string_view text) : s_(text) {}

  Value document() {
    Value root = makeTable();
    Value* current = &root;
    for (;;) {
      skipBlankLinesAndComments();
      if (eof()) break;
      if (peek() == '[') {
        current = header(root);
      } else {
        keyValue(*current);
      }
      endOfLine();
    }
    return root;
  }

 private:
  std::string_view s_;
  std::size_t pos_ = 0;
  int line_ = 1;

  [[noreturn]] void fail(const std::string& what) const {
    throw ParseError(std::format("line {}: {}", line_, what));
  }
  bool eof() const { return pos_ >= s_.size(); }
  char peek() const { return eof() ? '\0' : s_[pos_]; }
  char next() {
    const char c = s_[pos_++];
    if (c == '\n') ++line_;
    return c;
  }
  void skipSpaces() {
    while (!eof() && (peek() == ' ' || peek() == '\t')) next();
  }
  void skipComment() {
    if (peek() == '#') {
      while (!eof() && peek() != '\n') next();
    }
  }
  void skipBlankLinesAndComments() {
    for (;;) {
      skipSpaces();
      skipComment();
      if (!eof() && (peek() == '\n' || peek() == '\r')) {
        next();
        continue;
      }
      return;
    }
  }
  // Whitespace, newlines and comments inside arrays.
  void skipInsideArray() {
    for (;;) {
      skipSpaces();
      skipComment();
      if (!eof() && (peek() == '\n' || peek() == '\r')) {
        next();
        continue;
      }
      return;
    }
  }
  void endOfLine() {
    skipSpaces();
    skipComment();
    if (eof()) return;
    if (peek() == '\r') next();
    if (eof()) return;
    if (peek() != '\n') fail(std::format("unexpected '{}' after a value", peek()));
    next();
  }

  std::string bareKey() {
    std::string k;
    while (!eof() && (std::isalnum(static_cast<unsigned char>(peek())) || peek() == '_' || peek() == '-')) {
      k.push_back(next());
    }
    if (k.empty()) fail("expected a key");
    return k;
  }

  std::vector<std::string> dottedKey() {
    std::vector<std::string> parts;
    for (;;) {
      skipSpaces();
      if (peek() == '"') {
        parts.push_back(basicString());
      } else if (peek() == '\'') {
        parts.push_back(literalString());
      } else {
        parts.push_back(bareKey());
      }
      skipSpaces();
      if (peek() != '.') return parts;
      next();
    }
  }

  static Value* member(Value& table, const std::string& key) {
    for (auto& [k, v] : *table.table) {
      if (k == key) return &v;
    }
    return nullptr;
  }

  Value* descend(Value& from, const std::vector<std::string>& path, std::size_t count) {
    Value* at = &from;
    for (std::size_t i = 0; i < count; ++i) {
      Value* m = member(*at, path[i]);
      if (!m) {
        at->table->emplace_back(path[i], makeTable());
        m = &at->table->back().second;
      } else if (m->kind == Value::Kind::Array && m->array && !m->array->empty() &&
                 m->array->back().isTable()) {
        m = &m->array->back();  // the latest element of an array of tables
      } else if (!m->isTable()) {
        fail(std::format("'{}' is not a table", path[i]));
      }
      at = m;
    }
    return at;
  }

  Value* header(Value& root) {
    next();  // [
    const bool arrayOfTables = peek() == '[';
    if (arrayOfTables) next();
    const std::vector<std::string> path = dottedKey();
    if (peek() != ']') fail("expected ']' to close a table header");
    next();
    if (arrayOfTables) {
      if (peek() != ']') fail("expected ']]' to close an array-of-tables header");
      next();
    }
    Value* parent = descend(root, path, path.size() - 1);
    Value* m = member(*parent, path.back());
    if (arrayOfTables) {
      if (!m) {
        parent->table->emplace_back(path.back(), makeArray());
        m = &parent->table->back().second;
      } else if (!m->isArray()) {
        fail(std::format("'{}' is already defined as a non-array", path.back()));
      }
      m->array->push_back(makeTable());
      return &m->array->back();
    }
    if (!m) {
      parent->table->emplace_back(path.back(), makeTable());
      return &parent->table->back().second;
    }
    if (!m->isTable()) fail(std::format("'{}' is already defined", path.back()));
    return m;
  }

  void keyValue(Value& table) {
    const std::vector<std::string> path = dottedKey();
    skipSpaces();
    if (peek() != '=') fail("expected '=' after a key");
    next();
    skipSpaces();
    Value v = value();
    Value* parent = descend(table, path, path.size() - 1);
    if (member(*parent, path.back())) fail(std::format("duplicate key '{}'", path.back()));
    parent->table->emplace_back(path.back(), std::move(v));
  }

  std::string basicString() {
    next();  // "
    std::string out;
    for (;;) {
      if (eof() || peek() == '\n') fail("unterminated string");
      const char c = next();
      if (c == '"') return out;
      if (c != '\\') {
        out.push_back(c);
        continue;
      }
      if (eof()) fail("unterminated escape");
      const char e = next();
      switch (e) {
        case '"': out.push_back('"'); break;
        case '\\': out.push_back('\\'); break;
        case 'n': out.push_back('\n'); break;
        case 't': out.push_back('\t'); break;
        case 'r': out.push_back('\r'); break;
        case 'b': out.push_back('\b'); break;
        case 'f': out.push_back('\f'); break;
        case 'u': {
          unsigned code = 0;
          for (int i = 0; i < 4; ++i) {
            if (eof() || !std::isxdigit(static_cast<unsigned char>(peek()))) fail("bad \\u escape");
            const char h = next();
            code = code * 16 + static_cast<unsigned>(std::isdigit(static_cast<unsigned char>(h)) ? h - '0' : (std::tolower(h) - 'a' + 10));
          }
          if (code < 0x80) {
            out.push_back(static_cast<char>(code));
          } else if (code < 0x800) {
            out.push_back(static_cast<char>(0xC0 | (code >> 6)));
            out.push_back(static_cast<char>(0x80 | (code & 0x3F)));
          } else {
            out.push_back(static_cast<char>(0xE0 | (code >> 12)));
            out.push_back(static_cast<char>(0x80 | ((code >> 6) & 0x3F)));
            out.push_back(static_cast<char>(0x80 | (code & 0x3F)));
          }
          break;
        }
        default: fail(std::format("unknown escape '\\{}'", e));
      }
    }
  }

  std::string literalString() {
    next();  // '
    std::string out;
    for (;;) {
      if (eof() || peek() == '\n') fail("unterminated string");
      const char c = next();
      if (c == '\'') return out;
      out.push_back(c);
    }
  }

  Value number() {
    std::string tok;
    while (!eof()) {
      const char c = peek();
      if (std::isalnum(static_cast<unsigned char>(c)) || c == '+' || c == '-' || c == '.' || c == '_') {
        tok.push_back(next());
      } else {
        break;
      }
    }
    if (tok.empty()) fail("expected a value");
    if (tok == "true" || tok == "false") {
      Value v;
      v.kind = Value::Kind::Bool;
      v.boolean = tok == "true";
      return v;
    }
    std::string clean;
    for (const char c : tok) {
      if (c != '_') clean.push_back(c);
    }
    Value v;
    const std::string_view body = clean[0] == '+' || clean[0] == '-' ? std::string_view(clean).substr(1) : std::string_view(clean);
    if (body == "inf" || body == "nan") {
      v.kind = Value::Kind::Float;
      v.number = body == "inf" ? std::numeric_limits<double>::infinity() : std::numeric_limits<double>::quiet_NaN();
      if (clean[0] == '-') v.number = -v.number;
      return v;
    }
    const bool isFloat = clean.find_first_of(".eE") != std::string::npos &&
                         clean.rfind("0x", 0) != 0;
    char* end = nullptr;
    if (isFloat) {
      v.kind = Value::Kind::Float;
      v.number = std::strtod(clean.c_str(), &end);
    } else {
      v.kind = Value::Kind::Integer;
      v.integer = std::strtoll(clean.c_str(), &end, 10);
    }
    if (end == nullptr || *end != '\0') fail(std::format("malformed value '{}'", tok));
    return v;
  }

  Value arrayValue() {
    next();  // [
    Value v = makeArray();
    for (;;) {
      skipInsideArray();
      if (eof()) fail("unterminated array");
      if (peek() == ']') {
        next();
        return v;
      }
      v.array->push_back(value());
      skipInsideArray();
      if (peek() == ',') {
        next();
        continue;
      }
      skipInsideArray();
      if (peek() != ']') fail("expected ',' or ']' in an array");
    }
  }

  Value inlineTable() {
    next();  // {
    Value v = makeTable();
    skipSpaces();
    if (peek() == '}') {
      next();
      return v;
    }
    for (;;) {
      skipSpaces();
      keyValue(v);
      skipSpaces();
      if (peek() == ',') {
        next();
        continue;
      }
      if (peek() == '}') {
        next();
        return v;
      }
      fail("expected ',' or '}' in an inline table");
    }
  }

  Value value() {
    if (eof()) fail("expected a value");
    const char c = peek();
    if (c == '"') {
      Value v;
      v.kind = Value::Kind::String;
      v.str = basicString();
      return v;
    }
    if (c == '\'') {
      Value v;
      v.kind = Value::Kind::String;
      v.str = literalString();
      return v;
    }
    if (c == '[') return arrayValue();
    if (c == '{') return inlineTable();
    return number();
  }
};

}  // namespace

Value parse(std::string_view text) { return Parser(text).document(); }

}  // namespace spinsim::toml
