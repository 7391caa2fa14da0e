// opts.cpp -- opt-string parsing and option derivation for Super / Analyse (host).
//
//   parse_opt            crates/svpflow-core/src/params.rs:1-450 (lenient JSON: comments,
//                        bare keys, last duplicate wins, trailing data after an object)
//   super_opts_from_opt  crates/svpflow1/src/super_opts.rs:17-95
//   analyse_opts_*       crates/svpflow1/src/analyse_opts.rs:45-295, portable.rs:189-229
//   payload / header     crates/svpflow1/src/analyse_search.rs:2740-2841
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <utility>
#include <vector>

#include "svpf_internal.h"

namespace svpf {

struct OptValue {
    enum Kind { Object, Array, String, Number, Bool, Null } kind = Null;
    std::vector<std::pair<std::string, OptValue *>> members;  // Object
    std::vector<OptValue *> items;                             // Array
    std::string str;
    double num = 0.0;
    bool b = false;
    ~OptValue() {
        for (auto &m : members) delete m.second;
        for (auto *v : items) delete v;
    }
    // Value::get: the LAST member with this key wins (params.rs:77-85)
    const OptValue *get(const char *key) const {
        if (kind != Object) return nullptr;
        for (auto it = members.rbegin(); it != members.rend(); ++it)
            if (it->first == key) return it->second;
        return nullptr;
    }
};

OptTree::~OptTree() { delete root; }

namespace {

struct Parser {
    const unsigned char *s;
    size_t n, pos = 0;
    std::string err;

    int peek() const { return pos < n ? s[pos] : -1; }
    bool at2(const char *t) const { return pos + 2 <= n && s[pos] == (unsigned char)t[0] && s[pos + 1] == (unsigned char)t[1]; }
    bool consume(int c) {
        if (peek() == c) { pos++; return true; }
        return false;
    }
    void line_col(size_t p, size_t &line, size_t &col) const {
        line = 1;
        size_t line_start = 0, stop = p < n ? p : n, i = 0;
        while (i < stop) {
            if (s[i] == '\n') { line++; line_start = i + 1; }
            else if (s[i] == '\r') {
                line++;
                if (i + 1 < n && s[i + 1] == '\n') i++;
                line_start = i + 1;
            }
            i++;
        }
        col = stop - line_start + 1;
    }
    bool fail_at(size_t p, const char *msg) {
        size_t l, c;
        line_col(p, l, c);
        char buf[256];
        snprintf(buf, sizeof buf, "* Line %zu, Column %zu\n  %s\n", l, c, msg);
        err = buf;
        return false;
    }
    bool fail(const char *msg) { return fail_at(pos, msg); }
    void skip_space() {
        while (pos < n && (s[pos] == ' ' || s[pos] == '\n' || s[pos] == '\r' || s[pos] == '\t')) pos++;
    }
    void skip_ws() {  // params.rs:112-132
        for (;;) {
            skip_space();
            if (at2("//")) {
                pos += 2;
                while (pos < n && s[pos] != '\n' && s[pos] != '\r') pos++;
            } else if (at2("/*")) {
                pos += 2;
                while (!at2("*/")) {
                    if (pos >= n) return;
                    pos++;
                }
                pos += 2;
            } else {
                return;
            }
        }
    }
    bool skip_member_space() {  // params.rs:140-162: a comment before a member name is an error
        skip_space();
        if (at2("//")) {
            pos += 2;
            while (pos < n && s[pos] != '\n' && s[pos] != '\r') pos++;
            skip_space();
            return fail("Missing '}' or object member name");
        }
        if (at2("/*")) {
            pos += 2;
            while (!at2("*/")) {
                if (pos >= n) return fail("Missing '}' or object member name");
                pos++;
            }
            pos += 2;
            skip_space();
            return fail("Missing '}' or object member name");
        }
        return true;
    }
    bool value(OptValue *&out) {
        skip_ws();
        int c = peek();
        if (c == '{') return object(out);
        if (c == '[') return array(out);
        if (c == '"') {
            std::string t;
            if (!string(t)) return false;
            out = new OptValue;
            out->kind = OptValue::String;
            out->str = t;
            return true;
        }
        if (c == '-' || (c >= '0' && c <= '9')) return number(out);
        if (c == 't') return literal("true", OptValue::Bool, true, out);
        if (c == 'f') return literal("false", OptValue::Bool, false, out);
        if (c == 'n') return literal("null", OptValue::Null, false, out);
        return fail("Syntax error: value, object or array expected.");
    }
    bool literal(const char *lit, OptValue::Kind k, bool b, OptValue *&out) {
        size_t l = strlen(lit);
        if (pos + l <= n && memcmp(s + pos, lit, l) == 0) {
            pos += l;
            out = new OptValue;
            out->kind = k;
            out->b = b;
            return true;
        }
        return fail("invalid literal");
    }
    bool object(OptValue *&out) {
        pos++;  // '{'
        skip_ws();
        out = new OptValue;
        out->kind = OptValue::Object;
        if (consume('}')) return true;
        for (;;) {
            if (!skip_member_space()) return false;
            std::string key;
            if (peek() == '"') {
                if (!string(key)) return false;
            } else if (!identifier(key)) {
                return false;
            }
            skip_ws();
            if (!consume(':')) return fail("Missing ':' after object member name");
            OptValue *v = nullptr;
            if (!value(v)) return false;
            out->members.emplace_back(key, v);
            skip_ws();
            if (consume('}')) return true;
            if (!consume(',')) return fail("Missing ',' or '}' in object declaration");
        }
    }
    bool array(OptValue *&out) {
        pos++;  // '['
        skip_ws();
        out = new OptValue;
        out->kind = OptValue::Array;
        if (consume(']')) return true;
        for (;;) {
            OptValue *v = nullptr;
            if (!value(v)) return false;
            out->items.push_back(v);
            skip_ws();
            if (consume(']')) return true;
            if (!consume(',')) return fail("unexpected token");
        }
    }
    bool identifier(std::string &key) {
        size_t start = pos;
        int c = peek();
        if (!((c >= 'a' && c <= 'z') || (c >= 'A' && c <= 'Z') || c == '_'))
            return fail("Missing '}' or object member name");
        pos++;
        for (;;) {
            c = peek();
            if ((c >= 'a' && c <= 'z') || (c >= 'A' && c <= 'Z') || (c >= '0' && c <= '9') || c == '_') pos++;
            else break;
        }
        key.assign((const char *)s + start, pos - start);
        return true;
    }
    static void put_utf8(std::string &o, uint32_t cp) {
        if (cp < 0x80) o += (char)cp;
        else if (cp < 0x800) { o += (char)(0xC0 | (cp >> 6)); o += (char)(0x80 | (cp & 0x3F)); }
        else if (cp < 0x10000) {
            o += (char)(0xE0 | (cp >> 12)); o += (char)(0x80 | ((cp >> 6) & 0x3F)); o += (char)(0x80 | (cp & 0x3F));
        } else {
            o += (char)(0xF0 | (cp >> 18)); o += (char)(0x80 | ((cp >> 12) & 0x3F));
            o += (char)(0x80 | ((cp >> 6) & 0x3F)); o += (char)(0x80 | (cp & 0x3F));
        }
    }
    bool hex4(uint32_t &code) {
        code = 0;
        for (int i = 0; i < 4; i++) {
            int c = peek();
            if (c < 0) return false;
            pos++;
            uint32_t d;
            if (c >= '0' && c <= '9') d = (uint32_t)(c - '0');
            else if (c >= 'a' && c <= 'f') d = (uint32_t)(c - 'a' + 10);
            else if (c >= 'A' && c <= 'F') d = (uint32_t)(c - 'A' + 10);
            else return false;
            code = code * 16 + d;
        }
        return true;
    }
    bool string(std::string &out) {  // params.rs:240-324
        size_t start = pos;
        pos++;  // '"'
        std::string bytes;
        while (pos < n) {
            unsigned char c = s[pos++];
            if (c == '"') {
                out = bytes;
                return true;
            }
            if (c != '\\') { bytes += (char)c; continue; }
            int e = peek();
            if (e >= 0) pos++;
            switch (e) {
            case '"': bytes += '"'; break;
            case '\\': bytes += '\\'; break;
            case '/': bytes += '/'; break;
            case 'b': bytes += '\b'; break;
            case 'f': bytes += '\f'; break;
            case 'n': bytes += '\n'; break;
            case 'r': bytes += '\r'; break;
            case 't': bytes += '\t'; break;
            case 'u': {
                uint32_t code;
                if (!hex4(code)) return fail_at(start, "Bad unicode escape sequence in string: hexadecimal digit expected.");
                if (code >= 0xD800 && code <= 0xDBFF) {
                    uint32_t low;
                    if (!(consume('\\') && consume('u')) || !hex4(low) || !(low >= 0xDC00 && low <= 0xDFFF))
                        return fail_at(start, "additional six characters expected to parse unicode surrogate pair.");
                    put_utf8(bytes, 0x10000 + ((code - 0xD800) << 10) + (low - 0xDC00));
                } else if (code >= 0xDC00 && code <= 0xDFFF) {
                    put_utf8(bytes, 0xFFFD);
                } else {
                    put_utf8(bytes, code);
                }
                break;
            }
            default: return fail_at(start, "Bad escape sequence in string");
            }
        }
        return fail_at(start, "Syntax error: value, object or array expected.");
    }
    bool digits() {
        size_t st = pos;
        while (pos < n && s[pos] >= '0' && s[pos] <= '9') pos++;
        return pos != st;
    }
    bool number(OptValue *&out) {  // params.rs:326-366
        size_t start = pos;
        bool neg = consume('-');
        bool leading_dot = false;
        int c = peek();
        if (c >= '0' && c <= '9') {
            pos++;
            digits();
        } else if (neg && consume('.')) {
            if (!digits()) return fail_at(start, "is not a number.");
            leading_dot = true;
        } else if (neg) {
            out = new OptValue;
            out->kind = OptValue::Number;
            out->num = 0.0;
            return true;
        } else {
            return fail("invalid number");
        }
        if (!leading_dot && consume('.')) digits();
        if (consume('e') || consume('E')) {
            if (!consume('+')) consume('-');
            if (!digits()) return fail_at(start, "is not a number.");
        }
        std::string text((const char *)s + start, pos - start);
        if (leading_dot) text = "-0" + text.substr(1);
        out = new OptValue;
        out->kind = OptValue::Number;
        out->num = strtod(text.c_str(), nullptr);  // correctly rounded, like str::parse::<f64>
        return true;
    }
};

}  // namespace

bool parse_opt(const char *text, size_t len, OptTree &out, std::string &err) {
    delete out.root;
    out.root = nullptr;
    Parser p{(const unsigned char *)text, len};
    p.skip_ws();
    OptValue *v = nullptr;
    if (!p.value(v)) {
        delete v;
        err = p.err;
        return false;
    }
    p.skip_ws();
    if (p.pos == p.n || v->kind == OptValue::Object) {
        out.root = v;
        return true;
    }
    delete v;
    p.fail("extra data after JSON value");
    err = p.err;
    return false;
}

// ---------------------------------------------------------------- lookups (params.rs:23-75)
namespace {

const OptValue *at(const OptTree *t, std::initializer_list<const char *> path) {
    if (!t || !t->root) return nullptr;
    const OptValue *v = t->root;
    for (const char *k : path) {
        v = v->get(k);
        if (!v) return nullptr;
    }
    return v;
}
const OptValue *at_v(const OptValue *root, std::initializer_list<const char *> path) {
    const OptValue *v = root;
    for (const char *k : path) {
        if (!v) return nullptr;
        v = v->get(k);
    }
    return v;
}
bool int_of(const OptValue *v, int64_t &o) {
    if (!v) return false;
    switch (v->kind) {
    case OptValue::Number: {
        if (!isfinite(v->num)) return false;
        double t = trunc(v->num);
        if (t >= 9223372036854775808.0 || t < -9223372036854775808.0) return false;
        o = (int64_t)t;
        return true;
    }
    case OptValue::Bool: o = v->b ? 1 : 0; return true;
    case OptValue::Null: o = 0; return true;
    default: return false;
    }
}
bool bool_of(const OptValue *v, bool &o) {
    if (!v) return false;
    switch (v->kind) {
    case OptValue::Number: o = v->num != 0.0; return true;
    case OptValue::String: o = !v->str.empty(); return true;
    case OptValue::Object: o = !v->members.empty(); return true;
    case OptValue::Array: o = !v->items.empty(); return true;
    case OptValue::Bool: o = v->b; return true;
    case OptValue::Null: o = false; return true;
    }
    return false;
}
bool float_of(const OptValue *v, double &o) {
    if (!v) return false;
    switch (v->kind) {
    case OptValue::Number: o = v->num; return true;
    case OptValue::Bool: o = v->b ? 1.0 : 0.0; return true;
    case OptValue::Null: o = 0.0; return true;
    default: return false;
    }
}
int32_t as_i32(int64_t v) { return (int32_t)(uint32_t)(uint64_t)v; }
int32_t f64_as_i32(double x) {  // Rust `as i32`: saturating, NaN -> 0
    if (x != x) return 0;
    if (x >= 2147483647.0) return INT32_MAX;
    if (x <= -2147483648.0) return INT32_MIN;
    return (int32_t)x;
}
int32_t sat_mul_i32(int32_t a, int32_t b) {
    int64_t r = (int64_t)a * b;
    return r > INT32_MAX ? INT32_MAX : (r < INT32_MIN ? INT32_MIN : (int32_t)r);
}
int64_t geti(const OptTree *t, std::initializer_list<const char *> a, std::initializer_list<const char *> b, bool use_b,
             int64_t d) {
    int64_t v;
    if (int_of(at(t, a), v)) return v;
    if (use_b && int_of(at(t, b), v)) return v;
    return d;
}
bool getb(const OptTree *t, std::initializer_list<const char *> a, std::initializer_list<const char *> b, bool use_b,
          bool d) {
    bool v;
    if (bool_of(at(t, a), v)) return v;
    if (use_b && bool_of(at(t, b), v)) return v;
    return d;
}
double getf(const OptTree *t, std::initializer_list<const char *> a, std::initializer_list<const char *> b, double d) {
    double v;
    if (float_of(at(t, a), v)) return v;
    if (float_of(at(t, b), v)) return v;
    return d;
}
inline int32_t imax(int32_t a, int32_t b) { return a > b ? a : b; }
inline int32_t imin(int32_t a, int32_t b) { return a < b ? a : b; }
inline bool is_blk(int32_t n) { return n == 4 || n == 8 || n == 16 || n == 32; }

}  // namespace

// ---------------------------------------------------------------- super_opts.rs
int32_t reduce_dim(int32_t dim, int32_t n) {
    for (int32_t i = 0; i < n; i++) dim = 2 * (dim / 4);
    return dim;
}
int32_t auto_levels(int32_t width, int32_t height) {
    for (int32_t i = 0;; i++)
        if (reduce_dim(height, i) < 4 || reduce_dim(width, i) < 4) return i;
}
int32_t super_plane_height(int32_t base_h, int32_t pel, int32_t levels, bool full) {
    int32_t total = full ? pel * pel * base_h : 0;
    for (int32_t lv = 1; lv < levels; lv++) total += reduce_dim(base_h, lv);
    return total;
}
bool super_opts_from_opt(const OptTree *t, int32_t width, int32_t height, SuperOpts &o, std::string &err) {
    int32_t pel = as_i32(geti(t, {"pel"}, {}, false, 2));
    if (!(pel == 1 || pel == 2 || pel == 4)) { err = "SVSuper: pel has to be 1 or 2 or 4"; return false; }
    int32_t gpu = as_i32(geti(t, {"gpu"}, {}, false, 1));
    if (gpu < 0 || gpu > 2) { err = "SVSuper: gpu has to be 0 or 1 or 2"; return false; }
    int32_t scale_down = as_i32(geti(t, {"scale", "down"}, {}, false, 4));
    int32_t scale_up = as_i32(geti(t, {"scale", "up"}, {}, false, 2));
    if (gpu != 0) scale_up = 0;
    bool full = getb(t, {"full"}, {}, false, true);
    if (pel >= 2 && !full) { err = "SVSuper: can't ignore finest level with high pel value"; return false; }
    bool rc = getb(t, {"rc"}, {}, false, false);
    o.pel = pel; o.gpu = gpu; o.scale_down = scale_down; o.scale_up = scale_up;
    o.full = full; o.rc = rc; o.levels = auto_levels(width, height); o.width = width; o.height = height;
    return true;
}
int64_t super_pack_data(const SuperOpts &o) {
    uint64_t flags = o.rc ? 1 : 0;
    if (!o.full) flags |= 2;
    uint64_t raw = (uint64_t)(uint16_t)o.height | ((uint64_t)(uint16_t)o.width << 16) |
                   ((uint64_t)(uint8_t)o.pel << 32) | ((uint64_t)(uint8_t)o.levels << 40) |
                   ((uint64_t)(uint8_t)o.gpu << 48) | (flags << 56);
    return (int64_t)raw;
}

// ---------------------------------------------------------------- analyse_opts.rs
bool overlap_from_mode(int32_t bw, int32_t bh, int32_t mode, int32_t &ox, int32_t &oy, std::string &err) {
    switch (mode) {
    case 0: ox = 0; oy = 0; return true;
    case 1: ox = bw / 8; oy = bh / 8; return true;
    case 2: ox = bw / 4; oy = bh / 4; return true;
    case 3: ox = bw / 2; oy = bh / 2; return true;
    default:
        err = "SVAnalyse: overlap must be 0, 1 (=1/8*block), 2 (=1/4*block) or 3 (=1/2*block)";
        return false;
    }
}
int32_t auto_search_levels(int32_t w, int32_t h, int32_t bw, int32_t bh, int32_t ox, int32_t oy) {
    int32_t sx = imax(bw - ox, 1), sy = imax(bh - oy, 1);
    int32_t gw = imax((w - ox) / sx, 0), gh = imax((h - oy) / sy, 0);
    if (gw <= 0 || gh <= 0) return 1;
    int32_t end_x = ox + sx * gw, end_y = oy + sy * gh, levels = 0;
    for (;;) {
        int32_t gwl = ((end_x >> levels) - ox) / sx, ghl = ((end_y >> levels) - oy) / sy;
        if (gwl <= 0 || ghl <= 0) break;
        if (++levels > 12) break;
    }
    return imax(levels, 1);
}
bool analyse_opts_from_opt(const OptTree *t, int64_t sdata, const SuperOpts *hint, AnalyseOpts &o, std::string &err) {
    memset(&o, 0, sizeof(o));
    uint64_t r = (uint64_t)sdata;  // unpack_sdata, analyse_opts.rs:243-257
    int32_t height = (int32_t)(r & 0xFFFF), width = (int32_t)((r >> 16) & 0xFFFF);
    int32_t pel = (int32_t)((r >> 32) & 0xFF), slevels = (int32_t)((r >> 40) & 0xFF);
    int32_t selector = (int32_t)((r >> 48) & 0xFF);
    if (width <= 0 || height <= 0 || !(pel >= 1 && pel <= 4) || slevels <= 0) {
        if (!hint) { err = "SVAnalyse: invalid super clip params"; return false; }
        width = hint->width; height = hint->height; pel = hint->pel; slevels = hint->levels; selector = hint->gpu;
    }
    o.width = width; o.height = height; o.pel = pel; o.super_levels = slevels; o.selector = selector;
    int32_t vectors = as_i32(geti(t, {"vectors"}, {}, false, 3));
    if (vectors < 1 || vectors > 3) { err = "SVAnalyse: vectors must be 1, 2 or 3"; return false; }
    int32_t bw = as_i32(geti(t, {"block", "w"}, {}, false, 16));
    int32_t bh = as_i32(geti(t, {"block", "h"}, {}, false, bw));
    if (!is_blk(bw)) { err = "SVAnalyse: block.w must be 4/8/16/32"; return false; }
    int32_t om = as_i32(geti(t, {"block", "overlap"}, {}, false, 2));
    int32_t ox, oy;
    if (!overlap_from_mode(bw, bh, om, ox, oy, err)) return false;
    int32_t delta = as_i32(geti(t, {"special", "delta"}, {"delta"}, true, 1));
    double lambda = getf(t, {"main", "penalty", "lambda"}, {"penalty", "lambda"}, 10.0);
    int32_t lsad = as_i32(geti(t, {"main", "penalty", "lsad"}, {"penalty", "lsad"}, true, 8000));
    double plevel = fmax(getf(t, {"main", "penalty", "plevel"}, {"penalty", "plevel"}, 1.5), 0.01);
    o.pnew = as_i32(geti(t, {"main", "penalty", "pnew"}, {"penalty", "pnew"}, true, 50));
    o.pglobal = as_i32(geti(t, {"main", "penalty", "pglobal"}, {"penalty", "pglobal"}, true, 50));
    o.pzero = as_i32(geti(t, {"main", "penalty", "pzero"}, {"penalty", "pzero"}, true, 100));
    o.pnbour = as_i32(geti(t, {"main", "penalty", "pnbour"}, {"penalty", "pnbour"}, true, 50));
    o.prev = as_i32(geti(t, {"main", "penalty", "prev"}, {"penalty", "prev"}, true, 0));
    int32_t st = as_i32(geti(t, {"main", "search", "type"}, {"search", "type"}, true, 4));
    int32_t dist = as_i32(geti(t, {"main", "search", "distance"}, {"search", "distance"}, true, 2));
    o.coarse_search_type = as_i32(geti(t, {"main", "search", "coarse", "type"}, {"search", "coarse", "type"}, true, st));
    o.coarse_distance = as_i32(geti(t, {"main", "search", "coarse", "distance"}, {"search", "coarse", "distance"}, true, 0));
    o.coarse_trymany = getb(t, {"main", "search", "coarse", "trymany"}, {"search", "coarse", "trymany"}, true, false);
    int32_t cbs = as_i32(geti(t, {"main", "search", "coarse", "bad", "sad"}, {"search", "coarse", "bad", "sad"}, true, 1000));
    o.coarse_bad_range = as_i32(geti(t, {"main", "search", "coarse", "bad", "range"}, {}, false, -24));
    o.fine_satd = getb(t, {"main", "search", "satd"}, {"search", "satd"}, true, false);
    o.coarse_satd = getb(t, {"main", "search", "coarse", "satd"}, {}, false, true);
    o.sort = getb(t, {"main", "search", "sort"}, {"sort"}, true, true);
    const OptValue *ref_arr = at(t, {"refine"});  // analyse_opts.rs:150-164
    const OptValue *refine = (ref_arr && ref_arr->kind == OptValue::Array && !ref_arr->items.empty()) ? ref_arr->items[0] : nullptr;
    int64_t v;
    o.has_refine_thsad = 0;
    if (refine && int_of(at_v(refine, {"thsad"}), v)) {
        o.has_refine_thsad = 1;
        o.refine_thsad = as_i32(v) * imax((bw / 2) * (bh / 2), 1) / 32;
    }
    o.refine_search_type = (refine && int_of(at_v(refine, {"search", "type"}), v)) ? as_i32(v) : st;
    o.refine_distance = (refine && int_of(at_v(refine, {"search", "distance"}), v)) ? as_i32(v) : dist;
    bool rb;
    o.refine_satd = (refine && bool_of(at_v(refine, {"search", "satd"}), rb)) ? rb : o.fine_satd;
    int32_t levels = imax(imin(auto_search_levels(width, height, bw, bh, ox, oy), slevels), 1);
    if (int_of(at(t, {"main", "levels"}), v) && v > 0) levels = imax(imin(as_i32(v), slevels), 1);
    double area = (double)imax(bw * bh, 1);
    o.lambda = f64_as_i32(2.0 * area * 1000.0 * 0.015625 * lambda);
    int32_t area_scale = imax(bw * bh, 1) / 32;
    o.lsad = sat_mul_i32(lsad, area_scale);
    o.coarse_bad_sad = sat_mul_i32(cbs, area_scale);
    o.vectors = vectors; o.block_w = bw; o.block_h = bh; o.overlap_mode = om; o.overlap_x = ox; o.overlap_y = oy;
    o.delta = delta; o.levels = levels; o.plevel = plevel; o.search_type = st; o.distance = dist;
    return true;
}
bool analyse_opts_portable(const SuperOpts &so, int32_t bw, int32_t bh, int32_t om, int32_t vectors, AnalyseOpts &o,
                           std::string &err) {
    if (!is_blk(bw) || !is_blk(bh)) { err = "block dimensions must be 4, 8, 16 or 32"; return false; }
    if (vectors < 1 || vectors > 3) { err = "vectors must be 1, 2 or 3"; return false; }
    int32_t ox, oy;
    if (!overlap_from_mode(bw, bh, om, ox, oy, err)) return false;
    if (!analyse_opts_from_opt(nullptr, super_pack_data(so), &so, o, err)) return false;
    o.vectors = vectors; o.block_w = bw; o.block_h = bh; o.overlap_mode = om; o.overlap_x = ox; o.overlap_y = oy;
    o.levels = imax(imin(auto_search_levels(o.width, o.height, bw, bh, ox, oy), o.super_levels), 1);
    o.lambda = f64_as_i32((double)(bw * bh) * 312.5);
    return true;
}
void output_block(const AnalyseOpts &o, int32_t &bw, int32_t &bh, int32_t &ox, int32_t &oy) {
    if (o.has_refine_thsad) {
        bw = imax(o.block_w / 2, 4); bh = imax(o.block_h / 2, 4);
        ox = imax(o.overlap_x / 2, 0); oy = imax(o.overlap_y / 2, 0);
    } else {
        bw = o.block_w; bh = o.block_h; ox = o.overlap_x; oy = o.overlap_y;
    }
}
void output_grid(const AnalyseOpts &o, int32_t bw, int32_t bh, int32_t ox, int32_t oy, int32_t &gw, int32_t &gh) {
    int32_t sx = imax(bw - ox, 1), sy = imax(bh - oy, 1);
    gw = imax((o.width - ox) / sx, 1);
    gh = imax((o.height - oy) / sy, 1);
}
void level_grid(const AnalyseOpts &o, int32_t level, int32_t &gw, int32_t &gh) {
    int32_t sx = imax(o.block_w - o.overlap_x, 1), sy = imax(o.block_h - o.overlap_y, 1);
    int32_t gw0 = imax((o.width - o.overlap_x) / sx, 0), gh0 = imax((o.height - o.overlap_y) / sy, 0);
    int32_t end_x = o.overlap_x + sx * gw0, end_y = o.overlap_y + sy * gh0;
    gw = imax(((end_x >> level) - o.overlap_x) / sx, 1) + (level > 0);
    gh = imax(((end_y >> level) - o.overlap_y) / sy, 1) + (level > 0);
}
size_t payload_len(const AnalyseOpts &o) {
    int32_t bw, bh, ox, oy, gw, gh;
    output_block(o, bw, bh, ox, oy);
    output_grid(o, bw, bh, ox, oy, gw, gh);
    size_t nreg = (o.vectors == 1 || o.vectors == 2) ? 1 : 2;
    return 0x40 + nreg * (4 + (size_t)gw * gh * 8);
}
void vdata_header(const AnalyseOpts &o, int32_t h[16]) {
    int32_t bw, bh, ox, oy, gw, gh;
    output_block(o, bw, bh, ox, oy);
    output_grid(o, bw, bh, ox, oy, gw, gh);
    memset(h, 0, 16 * sizeof(int32_t));
    h[0] = 0xA0; h[1] = o.vectors == 1 ? 1 : (o.vectors == 2 ? 2 : 3); h[2] = bw; h[3] = bh; h[4] = o.pel;
    h[5] = o.has_refine_thsad ? 1 : o.levels; h[7] = o.width; h[8] = o.height; h[9] = ox; h[10] = oy;
    h[11] = gw; h[12] = gh; h[13] = o.selector; h[14] = o.delta;
}
SuperLayout portable_layout(const SuperOpts &so) { return strided_layout(so, so.width, so.width / 2); }

SuperLayout strided_layout(const SuperOpts &so, int64_t y_stride, int64_t c_stride) {
    SuperLayout L;
    L.width = so.width; L.height = so.height; L.pel = so.pel; L.levels = so.levels; L.full = so.full;
    L.super_h = super_plane_height(so.height, so.pel, so.levels, so.full);
    L.y_stride = y_stride;
    L.c_stride = c_stride;
    L.y_len = L.y_stride * (int64_t)L.super_h;
    L.c_len = L.c_stride * (int64_t)(L.super_h / 2);
    L.px_bytes = so.bits > 8 ? 2 : 1;
    L.frame_bytes = (L.y_len + 2 * L.c_len) * L.px_bytes;
    return L;
}

}  // namespace svpf
