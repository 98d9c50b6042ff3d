// Minimal JSON reader for the instance files: a small recursive-descent
// parser into a DOM.  Integers keep all 64 bits (the reference reads values
// with nlohmann's get<uint32_t>, which keeps the low 32 bits; masking to the
// word width here gives the same value).
#pragma once
#include <cstdint>
#include <cstdlib>
#include <map>
#include <memory>
#include <string>
#include <vector>

namespace simba {

struct JVal {
  enum Kind { NUL, BOOL, NUM, STR, ARR, OBJ } kind = NUL;
  bool b = false;
  bool is_int = false;
  uint64_t u = 0;  // integer value (two's complement for negatives)
  double d = 0.0;
  std::string s;
  std::vector<JVal> a;
  std::vector<std::pair<std::string, JVal>> o;

  const JVal* get(const std::string& key) const {
    for (auto& kv : o)
      if (kv.first == key) return &kv.second;
    return nullptr;
  }
};

class JParser {
 public:
  explicit JParser(const std::string& text) : t_(text) {}
  bool parse(JVal* out) {
    ws();
    if (!value(out, 0)) return false;
    ws();
    return i_ == t_.size();
  }
  std::string error() const { return "JSON parse error near byte " + std::to_string(i_); }

 private:
  void ws() {
    while (i_ < t_.size() && (t_[i_] == ' ' || t_[i_] == '\n' || t_[i_] == '\r' || t_[i_] == '\t')) ++i_;
  }
  bool lit(const char* w) {
    size_t n = std::char_traits<char>::length(w);
    if (t_.compare(i_, n, w) != 0) return false;
    i_ += n;
    return true;
  }
  bool value(JVal* v, int depth) {
    if (depth > 64 || i_ >= t_.size()) return false;
    char c = t_[i_];
    if (c == '{') return object(v, depth);
    if (c == '[') return array(v, depth);
    if (c == '"') {
      v->kind = JVal::STR;
      return str(&v->s);
    }
    if (c == 't') { v->kind = JVal::BOOL; v->b = true; return lit("true"); }
    if (c == 'f') { v->kind = JVal::BOOL; v->b = false; return lit("false"); }
    if (c == 'n') { v->kind = JVal::NUL; return lit("null"); }
    return number(v);
  }
  bool object(JVal* v, int depth) {
    v->kind = JVal::OBJ;
    ++i_;
    ws();
    if (i_ < t_.size() && t_[i_] == '}') { ++i_; return true; }
    for (;;) {
      ws();
      std::string key;
      if (i_ >= t_.size() || t_[i_] != '"' || !str(&key)) return false;
      ws();
      if (i_ >= t_.size() || t_[i_] != ':') return false;
      ++i_;
      ws();
      v->o.emplace_back(key, JVal());
      if (!value(&v->o.back().second, depth + 1)) return false;
      ws();
      if (i_ < t_.size() && t_[i_] == ',') { ++i_; continue; }
      if (i_ < t_.size() && t_[i_] == '}') { ++i_; return true; }
      return false;
    }
  }
  bool array(JVal* v, int depth) {
    v->kind = JVal::ARR;
    ++i_;
    ws();
    if (i_ < t_.size() && t_[i_] == ']') { ++i_; return true; }
    for (;;) {
      ws();
      v->a.emplace_back();
      if (!value(&v->a.back(), depth + 1)) return false;
      ws();
      if (i_ < t_.size() && t_[i_] == ',') { ++i_; continue; }
      if (i_ < t_.size() && t_[i_] == ']') { ++i_; return true; }
      return false;
    }
  }
  bool str(std::string* s) {
    ++i_;
    while (i_ < t_.size()) {
      char c = t_[i_++];
      if (c == '"') return true;
      if (c == '\\') {
        if (i_ >= t_.size()) return false;
        char e = t_[i_++];
        switch (e) {
          case 'n': s->push_back('\n'); break;
          case 't': s->push_back('\t'); break;
          case 'r': s->push_back('\r'); break;
          case 'b': s->push_back('\b'); break;
          case 'f': s->push_back('\f'); break;
          case 'u':
            if (i_ + 4 > t_.size()) return false;
            s->push_back('?');
            i_ += 4;
            break;
          default: s->push_back(e);
        }
      } else {
        s->push_back(c);
      }
    }
    return false;
  }
  bool number(JVal* v) {
    v->kind = JVal::NUM;
    size_t st = i_;
    bool neg = false;
    if (t_[i_] == '-') { neg = true; ++i_; }
    if (i_ >= t_.size() || t_[i_] < '0' || t_[i_] > '9') return false;
    unsigned __int128 acc = 0;
    bool overflow = false;
    while (i_ < t_.size() && t_[i_] >= '0' && t_[i_] <= '9') {
      acc = acc * 10 + (unsigned)(t_[i_] - '0');
      if (acc >> 64) overflow = true;
      ++i_;
    }
    bool frac = false;
    if (i_ < t_.size() && (t_[i_] == '.' || t_[i_] == 'e' || t_[i_] == 'E')) {
      frac = true;
      while (i_ < t_.size() && (isdigit((unsigned char)t_[i_]) || t_[i_] == '.' || t_[i_] == 'e' ||
                                t_[i_] == 'E' || t_[i_] == '+' || t_[i_] == '-'))
        ++i_;
    }
    v->d = strtod(t_.substr(st, i_ - st).c_str(), nullptr);
    if (!frac && !overflow) {
      v->is_int = true;
      uint64_t x = (uint64_t)acc;
      v->u = neg ? (uint64_t)(0 - x) : x;
    }
    return true;
  }
  const std::string& t_;
  size_t i_ = 0;
};

}  // namespace simba
