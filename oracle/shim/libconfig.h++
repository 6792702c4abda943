// Oracle test infrastructure only: a minimal, self-written stand-in for the libconfig++ API surface
// that the reference's ConfigSettings.cpp uses (Config::readFile, Config::lookup, Setting conversions,
// Setting::getLength / operator[], the four exception types). libconfig++ is not installed on this
// image, so the reference sources are compiled against this header to serve as the parity oracle.
//
// Grammar handled (libconfig syntax): `name = value` or `name : value` with optional `;`/`,`
// terminators, `//`, `#` and `/* */` comments, integers (decimal/hex, optional L suffix), floats
// (must contain '.', or an exponent), booleans (true/false, any case), strings (adjacent literals
// concatenate, \" \\ \n \t escapes), arrays [..], lists (..), groups {..} and dotted lookup paths.
// Types are strict, as in libconfig with auto-convert off: reading an int setting as double (or the
// reverse) throws SettingTypeException.
#ifndef ORACLE_SHIM_LIBCONFIG_HPP
#define ORACLE_SHIM_LIBCONFIG_HPP

#include <cctype>
#include <cstdlib>
#include <exception>
#include <fstream>
#include <memory>
#include <sstream>
#include <string>
#include <vector>

namespace libconfig {

class ConfigException : public std::exception {
 public:
  explicit ConfigException(std::string m) : msg_(std::move(m)) {}
  const char* what() const noexcept override { return msg_.c_str(); }

 private:
  std::string msg_;
};
class FileIOException : public ConfigException {
 public:
  using ConfigException::ConfigException;
};
class ParseException : public ConfigException {
 public:
  using ConfigException::ConfigException;
};
class SettingNotFoundException : public ConfigException {
 public:
  using ConfigException::ConfigException;
};
class SettingTypeException : public ConfigException {
 public:
  using ConfigException::ConfigException;
};

class Setting {
 public:
  enum Type { TypeNone, TypeInt, TypeFloat, TypeString, TypeBoolean, TypeGroup, TypeArray, TypeList };

  Type getType() const { return type_; }
  const std::string& getName() const { return name_; }
  int getLength() const { return static_cast<int>(children_.size()); }

  Setting& operator[](int i) const {
    if (i < 0 || i >= getLength())
      throw SettingNotFoundException(name_ + "[" + std::to_string(i) + "]");
    return *children_[static_cast<size_t>(i)];
  }
  Setting& operator[](const char* name) const {
    for (auto& c : children_)
      if (c->name_ == name) return *c;
    throw SettingNotFoundException(std::string(name));
  }
  bool exists(const char* name) const {
    for (auto& c : children_)
      if (c->name_ == name) return true;
    return false;
  }

  operator bool() const {
    if (type_ != TypeBoolean) throw SettingTypeException(name_);
    return b_;
  }
  operator int() const { return static_cast<int>(asInt()); }
  operator unsigned int() const { return static_cast<unsigned int>(asInt()); }
  operator long() const { return static_cast<long>(asInt()); }
  operator unsigned long() const { return static_cast<unsigned long>(asInt()); }
  operator long long() const { return asInt(); }
  operator unsigned long long() const { return static_cast<unsigned long long>(asInt()); }
  operator double() const {
    if (type_ != TypeFloat) throw SettingTypeException(name_);
    return f_;
  }
  operator float() const { return static_cast<float>(static_cast<double>(*this)); }
  operator const char*() const { return c_str(); }
  operator std::string() const { return std::string(c_str()); }
  const char* c_str() const {
    if (type_ != TypeString) throw SettingTypeException(name_);
    return s_.c_str();
  }

 private:
  friend class Config;
  friend struct ConfigParser;
  long long asInt() const {
    if (type_ != TypeInt) throw SettingTypeException(name_);
    return i_;
  }
  Type type_ = TypeNone;
  std::string name_;
  long long i_ = 0;
  double f_ = 0;
  bool b_ = false;
  std::string s_;
  std::vector<std::unique_ptr<Setting>> children_;
};

struct ConfigParser {
  const std::string& src;
  size_t pos = 0;
  int line = 1;
  explicit ConfigParser(const std::string& s) : src(s) {}

  [[noreturn]] void fail(const std::string& what) {
    throw ParseException("line " + std::to_string(line) + ": " + what);
  }
  void skip() {
    for (;;) {
      while (pos < src.size() && std::isspace(static_cast<unsigned char>(src[pos]))) {
        if (src[pos] == '\n') ++line;
        ++pos;
      }
      if (pos >= src.size()) return;
      if (src[pos] == '#' || (src[pos] == '/' && pos + 1 < src.size() && src[pos + 1] == '/')) {
        while (pos < src.size() && src[pos] != '\n') ++pos;
        continue;
      }
      if (src[pos] == '/' && pos + 1 < src.size() && src[pos + 1] == '*') {
        size_t e = src.find("*/", pos + 2);
        if (e == std::string::npos) fail("unterminated comment");
        for (size_t q = pos; q < e; ++q)
          if (src[q] == '\n') ++line;
        pos = e + 2;
        continue;
      }
      return;
    }
  }
  bool peek(char c) {
    skip();
    return pos < src.size() && src[pos] == c;
  }
  std::string name() {
    skip();
    size_t b = pos;
    if (pos >= src.size() || !(std::isalpha(static_cast<unsigned char>(src[pos])) || src[pos] == '*'))
      fail("expected a setting name");
    while (pos < src.size() &&
           (std::isalnum(static_cast<unsigned char>(src[pos])) || src[pos] == '_' || src[pos] == '-' || src[pos] == '*'))
      ++pos;
    return src.substr(b, pos - b);
  }
  void settings(Setting& group, char close) {
    for (;;) {
      skip();
      if (pos >= src.size()) {
        if (close) fail("unexpected end of file");
        return;
      }
      if (close && src[pos] == close) {
        ++pos;
        return;
      }
      auto s = std::make_unique<Setting>();
      s->name_ = name();
      skip();
      if (pos < src.size() && (src[pos] == '=' || src[pos] == ':'))
        ++pos;
      else
        fail("expected '=' or ':' after " + s->name_);
      value(*s);
      skip();
      if (pos < src.size() && (src[pos] == ';' || src[pos] == ',')) ++pos;
      group.children_.push_back(std::move(s));
    }
  }
  void value(Setting& s) {
    skip();
    if (pos >= src.size()) fail("missing value");
    char c = src[pos];
    if (c == '{') {
      ++pos;
      s.type_ = Setting::TypeGroup;
      settings(s, '}');
    } else if (c == '[' || c == '(') {
      char close = c == '[' ? ']' : ')';
      ++pos;
      s.type_ = c == '[' ? Setting::TypeArray : Setting::TypeList;
      skip();
      if (peek(close)) {
        ++pos;
        return;
      }
      for (;;) {
        auto e = std::make_unique<Setting>();
        e->name_ = s.name_;
        value(*e);
        s.children_.push_back(std::move(e));
        skip();
        if (peek(',')) {
          ++pos;
          continue;
        }
        if (peek(close)) {
          ++pos;
          return;
        }
        fail("expected ',' or closing bracket");
      }
    } else if (c == '"') {
      s.type_ = Setting::TypeString;
      while (peek('"')) {
        ++pos;
        while (pos < src.size() && src[pos] != '"') {
          if (src[pos] == '\\' && pos + 1 < src.size()) {
            char e = src[++pos];
            s.s_ += e == 'n' ? '\n' : e == 't' ? '\t' : e;
          } else {
            s.s_ += src[pos];
          }
          ++pos;
        }
        if (pos >= src.size()) fail("unterminated string");
        ++pos;
      }
    } else {
      size_t b = pos;
      while (pos < src.size() && (std::isalnum(static_cast<unsigned char>(src[pos])) || src[pos] == '.' ||
                                  src[pos] == '+' || src[pos] == '-' || src[pos] == '_'))
        ++pos;
      std::string tok = src.substr(b, pos - b);
      if (tok.empty()) fail("bad value");
      std::string low;
      for (char ch : tok) low += static_cast<char>(std::tolower(static_cast<unsigned char>(ch)));
      if (low == "true" || low == "false") {
        s.type_ = Setting::TypeBoolean;
        s.b_ = low == "true";
        return;
      }
      bool hex = low.size() > 2 && (low.rfind("0x", 0) == 0 || low.rfind("-0x", 0) == 0);
      bool isFloat = !hex && (low.find('.') != std::string::npos || low.find('e') != std::string::npos);
      char* end = nullptr;
      if (isFloat) {
        s.type_ = Setting::TypeFloat;
        s.f_ = std::strtod(tok.c_str(), &end);
      } else {
        s.type_ = Setting::TypeInt;
        s.i_ = std::strtoll(tok.c_str(), &end, hex ? 16 : 10);
        while (end && (*end == 'L' || *end == 'l')) ++end;
      }
      if (!end || *end != '\0') fail("bad number '" + tok + "'");
    }
  }
};

class Config {
 public:
  Config() { root_.type_ = Setting::TypeGroup; }
  void readFile(const char* filename) {
    std::ifstream in(filename);
    if (!in) throw FileIOException("cannot open " + std::string(filename));
    std::stringstream ss;
    ss << in.rdbuf();
    readString(ss.str());
  }
  void readString(const std::string& text) {
    Setting fresh;
    fresh.type_ = Setting::TypeGroup;
    ConfigParser p(text);
    p.settings(fresh, 0);
    root_.children_ = std::move(fresh.children_);
  }
  Setting& lookup(const char* path) const {
    const Setting* cur = &root_;
    std::string p(path);
    size_t b = 0;
    for (;;) {
      size_t e = p.find('.', b);
      std::string part = p.substr(b, e == std::string::npos ? std::string::npos : e - b);
      if (!cur->exists(part.c_str())) throw SettingNotFoundException(p);
      cur = &(*cur)[part.c_str()];
      if (e == std::string::npos) break;
      b = e + 1;
    }
    return const_cast<Setting&>(*cur);
  }
  bool exists(const char* path) const {
    try {
      lookup(path);
      return true;
    } catch (const SettingNotFoundException&) {
      return false;
    }
  }
  Setting& getRoot() const { return const_cast<Setting&>(root_); }

 private:
  Setting root_;
};

}  // namespace libconfig

#endif
