// vah_properties.cpp -- see vah_properties.h.
#include "vah_properties.h"

#include <cctype>
#include <cerrno>
#include <cstdio>
#include <cstdlib>

namespace vah {

namespace {

struct Cursor {
    const std::string &t;
    size_t p = 0;
    int line = 1;
    explicit Cursor(const std::string &s) : t(s) {}
    bool eof() const { return p >= t.size(); }
    char peek(size_t k = 0) const { return p + k < t.size() ? t[p + k] : '\0'; }
    void adv() {
        if (t[p] == '\n') ++line;
        ++p;
    }
};

// Skip blanks and the three comment forms.
void skip(Cursor &c) {
    while (!c.eof()) {
        char ch = c.peek();
        if (std::isspace((unsigned char)ch)) {
            c.adv();
        } else if (ch == '#' || (ch == '/' && c.peek(1) == '/')) {
            while (!c.eof() && c.peek() != '\n') c.adv();
        } else if (ch == '/' && c.peek(1) == '*') {
            c.adv();
            c.adv();
            while (!c.eof() && !(c.peek() == '*' && c.peek(1) == '/')) c.adv();
            if (!c.eof()) {
                c.adv();
                c.adv();
            }
        } else {
            break;
        }
    }
}

bool is_name_start(char ch) { return std::isalpha((unsigned char)ch) || ch == '*'; }
bool is_name_char(char ch) { return std::isalnum((unsigned char)ch) || ch == '_' || ch == '-' || ch == '*'; }

std::string fail(const Cursor &c, const std::string &what) {
    char buf[64];
    std::snprintf(buf, sizeof(buf), " at line %d", c.line);
    return what + buf;
}

bool parse_scalar(Cursor &c, Setting *out, std::string *err) {
    char ch = c.peek();
    if (ch == '"') {
        out->type = Setting::STRING;
        out->s.clear();
        while (c.peek() == '"') {  // adjacent literals concatenate
            c.adv();
            while (!c.eof() && c.peek() != '"') {
                if (c.peek() == '\\' && c.p + 1 < c.t.size()) {
                    c.adv();
                    char e = c.peek();
                    out->s += e == 'n' ? '\n' : e == 't' ? '\t' : e == 'r' ? '\r' : e;
                } else {
                    out->s += c.peek();
                }
                c.adv();
            }
            if (c.eof()) {
                *err = fail(c, "unterminated string");
                return false;
            }
            c.adv();
            skip(c);
        }
        return true;
    }
    // bare word: number or boolean
    size_t start = c.p;
    while (!c.eof() && !std::isspace((unsigned char)c.peek()) && c.peek() != ';' && c.peek() != ',' &&
           c.peek() != '#' && !(c.peek() == '/' && (c.peek(1) == '/' || c.peek(1) == '*')))
        c.adv();
    std::string w = c.t.substr(start, c.p - start);
    std::string lw;
    for (char x : w) lw += (char)std::tolower((unsigned char)x);
    if (lw == "true" || lw == "false") {
        out->type = Setting::BOOL;
        out->b = lw == "true";
        return true;
    }
    if (w.empty()) {
        *err = fail(c, "missing value");
        return false;
    }
    const bool hex = lw.size() > 2 && (lw.compare(0, 2, "0x") == 0 || lw.compare(0, 3, "-0x") == 0 ||
                                       lw.compare(0, 3, "+0x") == 0);
    const bool is_float = !hex && (lw.find('.') != std::string::npos || lw.find('e') != std::string::npos);
    errno = 0;
    char *end = nullptr;
    if (is_float) {
        out->type = Setting::FLOAT;
        out->f = std::strtod(w.c_str(), &end);
    } else {
        std::string digits = w;
        if (!digits.empty() && (digits.back() == 'L' || digits.back() == 'l')) digits.pop_back();
        if (!digits.empty() && (digits.back() == 'L' || digits.back() == 'l')) digits.pop_back();
        out->type = Setting::INT;
        out->i = std::strtoll(digits.c_str(), &end, 0);
        if (end && *end == '\0') return errno == 0 || (*err = fail(c, "integer out of range"), false);
        *err = fail(c, "malformed number '" + w + "'");
        return false;
    }
    if (!end || *end != '\0' || errno) {
        *err = fail(c, "malformed number '" + w + "'");
        return false;
    }
    return true;
}

// Skip a group/array/list value (not used by the reference's files).
bool skip_aggregate(Cursor &c, std::string *err) {
    int depth = 0;
    do {
        char ch = c.peek();
        if (ch == '{' || ch == '[' || ch == '(') ++depth;
        if (ch == '}' || ch == ']' || ch == ')') --depth;
        if (ch == '"') {
            Setting tmp;
            if (!parse_scalar(c, &tmp, err)) return false;
            continue;
        }
        c.adv();
    } while (depth > 0 && !c.eof());
    if (depth != 0) {
        *err = fail(c, "unbalanced brackets");
        return false;
    }
    return true;
}

}  // namespace

bool Properties::read_string(const std::string &text, std::string *err) {
    map_.clear();
    Cursor c(text);
    std::string dummy;
    if (!err) err = &dummy;
    for (;;) {
        skip(c);
        if (c.eof()) return true;
        if (!is_name_start(c.peek())) {
            *err = fail(c, "syntax error");
            return false;
        }
        size_t s0 = c.p;
        while (!c.eof() && is_name_char(c.peek())) c.adv();
        std::string name = c.t.substr(s0, c.p - s0);
        skip(c);
        if (c.peek() != '=' && c.peek() != ':') {
            *err = fail(c, "expected '=' after " + name);
            return false;
        }
        c.adv();
        skip(c);
        char ch = c.peek();
        if (ch == '{' || ch == '[' || ch == '(') {
            if (!skip_aggregate(c, err)) return false;
        } else {
            Setting st;
            if (!parse_scalar(c, &st, err)) return false;
            map_[name] = st;
        }
        skip(c);
        if (c.peek() == ';' || c.peek() == ',') c.adv();
    }
}

bool Properties::read_file(const std::string &path, std::string *err) {
    FILE *fp = std::fopen(path.c_str(), "rb");
    if (!fp) {
        if (err) *err = "file I/O error";
        map_.clear();
        return false;
    }
    std::string text;
    char buf[4096];
    size_t n;
    while ((n = std::fread(buf, 1, sizeof(buf), fp)) > 0) text.append(buf, n);
    std::fclose(fp);
    return read_string(text, err);
}

bool Properties::lookup_int(const std::string &name, int *out) const {
    auto it = map_.find(name);
    if (it == map_.end()) return false;
    const Setting &s = it->second;
    if (s.type == Setting::INT) {
        *out = (int)s.i;
        return true;
    }
    if (s.type == Setting::FLOAT && auto_convert) {
        *out = (int)s.f;
        return true;
    }
    return false;
}

bool Properties::lookup_float(const std::string &name, double *out) const {
    auto it = map_.find(name);
    if (it == map_.end()) return false;
    const Setting &s = it->second;
    if (s.type == Setting::FLOAT) {
        *out = s.f;
        return true;
    }
    if (s.type == Setting::INT && auto_convert) {
        *out = (double)s.i;
        return true;
    }
    return false;
}

bool Properties::lookup_bool(const std::string &name, bool *out) const {
    auto it = map_.find(name);
    if (it == map_.end() || it->second.type != Setting::BOOL) return false;
    *out = it->second.b;
    return true;
}

bool Properties::lookup_string(const std::string &name, std::string *out) const {
    auto it = map_.find(name);
    if (it == map_.end() || it->second.type != Setting::STRING) return false;
    *out = it->second.s;
    return true;
}

}  // namespace vah
