// yaml_lite.hpp -- the YAML subset of the tdse input files (inp/*.yaml in the
// reference, read there with yaml-cpp, src/tdse/td_read.cpp:3-47): top-level
// sections, one level of `key: value` below them, scalars (plain, "double"
// or 'single' quoted), flow sequences [a, b, c], and # comments.
#pragma once
#include <fstream>
#include <map>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

namespace yl {

struct Error : std::runtime_error {
  using std::runtime_error::runtime_error;
};

class Doc {
 public:
  static Doc load(const std::string& path) {
    std::ifstream in(path);
    if (!in) throw Error("yaml: cannot open " + path);
    Doc d;
    std::string line, section;
    int lineno = 0;
    while (std::getline(in, line)) {
      ++lineno;
      const std::string body = strip_comment(line);
      if (trim(body).empty()) continue;
      const size_t indent = body.find_first_not_of(' ');
      const size_t colon = find_colon(body);
      if (colon == std::string::npos) throw Error("yaml: line " + std::to_string(lineno) + ": no ':'");
      const std::string key = trim(body.substr(indent, colon - indent));
      const std::string val = trim(body.substr(colon + 1));
      if (indent == 0) {
        section = key;
        if (!val.empty()) d.v_[""][key] = unquote(val);
        d.v_[section];
      } else {
        if (section.empty()) throw Error("yaml: indented key outside a section");
        d.v_[section][key] = val;
      }
    }
    return d;
  }
  bool has(const std::string& sec, const std::string& key) const {
    auto s = v_.find(sec);
    return s != v_.end() && s->second.count(key);
  }
  std::string raw(const std::string& sec, const std::string& key) const {
    auto s = v_.find(sec);
    if (s == v_.end() || !s->second.count(key))
      throw Error("yaml: missing " + sec + "." + key);
    return s->second.at(key);
  }
  std::string str(const std::string& sec, const std::string& key) const {
    return unquote(raw(sec, key));
  }
  double num(const std::string& sec, const std::string& key) const {
    const std::string s = str(sec, key);
    size_t pos = 0;
    double v;
    try {
      v = std::stod(s, &pos);
    } catch (...) {
      throw Error("yaml: " + sec + "." + key + " is not a number: " + s);
    }
    if (pos != s.size()) throw Error("yaml: " + sec + "." + key + " is not a number: " + s);
    return v;
  }
  int integer(const std::string& sec, const std::string& key) const {
    const std::string s = str(sec, key);
    size_t pos = 0;
    int v;
    try {
      v = std::stoi(s, &pos);
    } catch (...) {
      throw Error("yaml: " + sec + "." + key + " is not an integer: " + s);
    }
    if (pos != s.size()) throw Error("yaml: " + sec + "." + key + " is not an integer: " + s);
    return v;
  }
  std::vector<int> int_list(const std::string& sec, const std::string& key) const {
    std::string s = trim(raw(sec, key));
    if (s.size() < 2 || s.front() != '[' || s.back() != ']')
      throw Error("yaml: " + sec + "." + key + " is not a [list]");
    s = s.substr(1, s.size() - 2);
    std::vector<int> out;
    std::stringstream ss(s);
    std::string item;
    while (std::getline(ss, item, ',')) {
      item = trim(item);
      if (item.empty()) continue;
      out.push_back(std::stoi(item));
    }
    return out;
  }

 private:
  std::map<std::string, std::map<std::string, std::string>> v_;

  static std::string trim(const std::string& s) {
    const size_t a = s.find_first_not_of(" \t\r");
    if (a == std::string::npos) return "";
    const size_t b = s.find_last_not_of(" \t\r");
    return s.substr(a, b - a + 1);
  }
  static std::string strip_comment(const std::string& s) {
    char q = 0;
    for (size_t i = 0; i < s.size(); ++i) {
      const char c = s[i];
      if (q) {
        if (c == q) q = 0;
      } else if (c == '"' || c == '\'') {
        q = c;
      } else if (c == '#') {
        return s.substr(0, i);
      }
    }
    return s;
  }
  static size_t find_colon(const std::string& s) {
    char q = 0;
    for (size_t i = 0; i < s.size(); ++i) {
      const char c = s[i];
      if (q) {
        if (c == q) q = 0;
      } else if (c == '"' || c == '\'') {
        q = c;
      } else if (c == ':') {
        return i;
      }
    }
    return std::string::npos;
  }
  static std::string unquote(const std::string& s0) {
    const std::string s = trim(s0);
    if (s.size() >= 2 && ((s.front() == '"' && s.back() == '"') || (s.front() == '\'' && s.back() == '\'')))
      return s.substr(1, s.size() - 2);
    return s;
  }
};

}  // namespace yl
