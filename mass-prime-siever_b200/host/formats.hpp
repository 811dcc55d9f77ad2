// formats.hpp -- the file formats of the siever's host surface.
//
// The B200 worker keeps the reference program's files so that a user can
// swap it in: prime.ini and worktodo.txt in, relations.p, core_<id>.p and
// results.json out, and the same log line layout.  This header implements
// them from the specification below (the byte-level behaviour is the
// interface; the implementation is this project's own).
//
// Log line:     "<YYYY-MM-DD HH:MM:SS> UTC+0 [<LEVEL>] <message>" (UTC), to
//               stderr and appended to siever.log (Logger.hpp:15-29, 143-155).
//               A FATAL line ends the program with exit status 1.
//
// prime.ini:    text lines; surrounding white space ignored; blank lines and
//               lines starting with '#' skipped; otherwise "key=value" split
//               at the first '=' (both sides trimmed, empty key skipped,
//               unknown keys ignored, a later line overrides an earlier one).
//               Integer keys take std::stoi's reading (leading digits after an
//               optional sign; no digits is an error).  Keys and defaults
//               (Config.hpp:16-26): CPU_count (detected cores), MemoryAllowed
//               (10240, MB), UseGPU (0), GPU_device (0), GPU_backend ("auto"),
//               GPU_threads (2, at least 1), GPU_sieve (0), GPU_classes (1),
//               GPU_strict (0).  CPU_count = 0 is kept only together with a
//               nonzero UseGPU (GPU-only sieving); otherwise a value <= 0 means
//               "detect".  MemoryAllowed <= 0 means 10240.  When the file is
//               missing, or CPU_count or MemoryAllowed was absent or replaced,
//               the file is rewritten with exactly four lines CPU_count=,
//               MemoryAllowed=, UseGPU=, GPU_device= and an INFO line says so
//               (Config.hpp:50-122).
//
// worktodo.txt: one item per line; blank and '#' lines skipped; an optional
//               "Factor=" prefix; fields separated by ',' (white space around
//               a field ignored, empty fields dropped); exactly 6 fields
//               b,c,P0,P1,N0,N1 or 8 with mod,res.  b..N1 are signed 128-bit
//               integers written in decimal, or hexadecimal after "0x", or
//               octal after a leading "0" (the string reading of the
//               reference's 128-bit type); mod and res are std::stoull
//               readings.  Errors (fatal, "worktodo line <k> ..."): wrong field
//               count, a number that does not parse or mod = 0 or res >= mod
//               ("parse error: ..."), P0 >= P1, N0 >= N1, N1 - N0 > 10^7; no
//               item at all: "No work items found in <path>"
//               (Config.hpp:124-200).
//
// relations.p / core_<id>.p: one relation per line, "p, M, q\n" written as
//               "%llu, %llu, %llu\n" (Worker.hpp:294-297).  Read back as three
//               unsigned integers separated by ',' with white space allowed
//               before each token; anything after q is ignored; blank lines are
//               skipped; any other line is fatal "Malformed relation line: <line>"
//               (Worker.hpp:497-525).
//
// Candidates:   for the item's n in [N0, N1), the primes p of the relations
//               with n == M (mod q), in relation order (Worker.hpp:527-559).
//               p is not listed for n when b^n + c == p, where b^n is built by
//               repeated multiplication that gives up (no skip) as soon as the
//               running power exceeds 2p -- the reference's exact test.
//
// results.json: a JSON array; each finished item appends one object with the
//               keys, in order, Timestamp (the log's timestamp), b, c, P0 (the
//               item's original P0, before any resume), P1, N0, N1, prp (the
//               in-class n with no candidate prime, ascending) and factored
//               (objects {"n": n, "factors": [p, ...]} for the other in-class
//               n).  Integers outside int64 are written as decimal strings.
//               The whole file is re-written compactly (no white space) with a
//               final '\n', existing entries re-serialised the way
//               boost::json::serialize writes them; an existing file that is
//               not one JSON array is fatal (Results.hpp:57-140).
#pragma once

#include <cerrno>
#include <cctype>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <ctime>
#include <fstream>
#include <iostream>
#include <mutex>
#include <stdexcept>
#include <string>
#include <unistd.h>
#include <utility>
#include <vector>

namespace mpsio {

typedef __int128 i128;
typedef unsigned __int128 u128;

// ------------------------------------------------------------------ text --

inline bool is_space(char ch) { return std::isspace((unsigned char)ch) != 0; }

// The text without its leading and trailing white space.
inline std::string strip(const std::string& s) {
    size_t a = 0, b = s.size();
    while (a < b && is_space(s[a])) ++a;
    while (b > a && is_space(s[b - 1])) --b;
    return s.substr(a, b - a);
}

inline std::string i128_text(i128 v) {
    char buf[48];
    int k = (int)sizeof(buf);
    buf[--k] = '\0';
    u128 m = v < 0 ? (u128)0 - (u128)v : (u128)v;
    do {
        buf[--k] = (char)('0' + (int)(m % 10));
        m /= 10;
    } while (m != 0);
    if (v < 0) buf[--k] = '-';
    return std::string(buf + k);
}

// A signed 128-bit integer as the reference's 128-bit type reads a string:
// an optional '-', then "0x"/"0X" and hex digits, or "0" and octal digits, or
// decimal digits (no digits after the prefix reads as 0); any other
// character is an error.  Values beyond 128 bits are an error here.
inline i128 i128_parse(const std::string& text) {
    const char* s = text.c_str();
    const bool neg = *s == '-';
    if (neg) ++s;
    unsigned radix = 10;
    if (s[0] == '0' && (s[1] == 'x' || s[1] == 'X')) {
        radix = 16;
        s += 2;
    } else if (s[0] == '0') {
        radix = 8;
        ++s;
    }
    const u128 limit = (u128)1 << 127;                 // |value| <= 2^127 (only -2^127 reaches it)
    u128 mag = 0;
    for (; *s; ++s) {
        const char ch = *s;
        unsigned d;
        if (ch >= '0' && ch <= '9') d = (unsigned)(ch - '0');
        else if (ch >= 'a' && ch <= 'f') d = 10u + (unsigned)(ch - 'a');
        else if (ch >= 'A' && ch <= 'F') d = 10u + (unsigned)(ch - 'A');
        else d = 99;
        if (d >= radix) throw std::invalid_argument("Unexpected content found while parsing character string.");
        if (mag > (limit - d) / radix) throw std::out_of_range("\"" + text + "\" does not fit in 128 bits");
        mag = mag * radix + d;
    }
    if (!neg && mag == limit) throw std::out_of_range("\"" + text + "\" does not fit in 128 bits");
    return neg ? (i128)((u128)0 - mag) : (i128)mag;
}

// std::stoi / std::stoull readings (leading white space, sign, decimal
// digits, the rest ignored), throwing what those functions throw.
inline int int_reading(const std::string& s) {
    const char* b = s.c_str();
    char* e = nullptr;
    errno = 0;
    const long v = std::strtol(b, &e, 10);
    if (e == b) throw std::invalid_argument("stoi");
    if (errno == ERANGE || v < INT32_MIN || v > INT32_MAX) throw std::out_of_range("stoi");
    return (int)v;
}

inline uint64_t u64_reading(const std::string& s) {
    const char* b = s.c_str();
    char* e = nullptr;
    errno = 0;
    const unsigned long long v = std::strtoull(b, &e, 10);
    if (e == b) throw std::invalid_argument("stoull");
    if (errno == ERANGE) throw std::out_of_range("stoull");
    return v;
}

// ----------------------------------------------------------------- log --

inline std::string utc_stamp(std::time_t t) {
    std::tm tm{};
    gmtime_r(&t, &tm);
    char buf[48];
    std::strftime(buf, sizeof(buf), "%Y-%m-%d %H:%M:%S UTC+0", &tm);
    return buf;
}
inline std::string utc_now() { return utc_stamp(std::time(nullptr)); }

class Log {
public:
    static Log& get() {
        static Log one;
        return one;
    }
    void open(const std::string& path) {
        std::lock_guard<std::mutex> g(mu_);
        if (file_.is_open()) return;
        file_.open(path, std::ios::app);
        if (!file_) throw std::runtime_error("Failed to open log file: " + path);
    }
    void line(const char* level, const std::string& msg) {
        std::string text = utc_now();
        text.append(" [").append(level).append("] ").append(msg);
        std::lock_guard<std::mutex> g(mu_);
        std::cerr << text << std::endl;
        if (file_.is_open()) file_ << text << std::endl;
    }

private:
    std::mutex mu_;
    std::ofstream file_;
};

inline void info(const std::string& m) { Log::get().line("INFO", m); }
[[noreturn]] inline void fatal(const std::string& m) {
    Log::get().line("FATAL", m);
    std::exit(1);
}

// ------------------------------------------------------------- prime.ini --

struct PrimeConfig {
    int cpu_count = 0;
    int memory_allowed_mb = 10240;
    int use_gpu = 0;
    int gpu_device = 0;
    std::string gpu_backend = "auto";
    int gpu_threads = 2;
    int gpu_sieve = 0;
    int gpu_classes = 1;
    int gpu_strict = 0;
};

inline int cores_detected() {
    const long n = sysconf(_SC_NPROCESSORS_ONLN);
    return n > 0 ? (int)n : 1;
}

// (key, value) pairs of an ini file in file order; *exists tells whether it was there.
inline std::vector<std::pair<std::string, std::string>> ini_pairs(const std::string& path, bool* exists) {
    std::vector<std::pair<std::string, std::string>> kv;
    std::ifstream in(path);
    *exists = (bool)in;
    for (std::string raw; std::getline(in, raw);) {
        const std::string s = strip(raw);
        if (s.empty() || s[0] == '#') continue;
        const size_t eq = s.find('=');
        if (eq == std::string::npos) continue;
        std::string key = strip(s.substr(0, eq));
        if (!key.empty()) kv.emplace_back(std::move(key), strip(s.substr(eq + 1)));
    }
    return kv;
}

inline PrimeConfig read_prime_ini(const std::string& path) {
    PrimeConfig cfg;
    cfg.cpu_count = cores_detected();
    struct IntKey {
        const char* name;
        int PrimeConfig::*field;
        int floor;          // values below are raised to this (INT32_MIN: none)
    };
    static const IntKey keys[] = {
        {"CPU_count", &PrimeConfig::cpu_count, INT32_MIN},     {"MemoryAllowed", &PrimeConfig::memory_allowed_mb, INT32_MIN},
        {"UseGPU", &PrimeConfig::use_gpu, INT32_MIN},          {"GPU_device", &PrimeConfig::gpu_device, INT32_MIN},
        {"GPU_threads", &PrimeConfig::gpu_threads, 1},         {"GPU_sieve", &PrimeConfig::gpu_sieve, INT32_MIN},
        {"GPU_classes", &PrimeConfig::gpu_classes, INT32_MIN}, {"GPU_strict", &PrimeConfig::gpu_strict, INT32_MIN},
    };
    bool exists = false, saw_cpu = false, saw_mem = false;
    for (const auto& [key, value] : ini_pairs(path, &exists)) {
        if (key == "GPU_backend") {
            cfg.gpu_backend = value;
            continue;
        }
        for (const IntKey& k : keys) {
            if (key != k.name) continue;
            const int v = int_reading(value);
            cfg.*(k.field) = v < k.floor ? k.floor : v;
            saw_cpu |= k.field == &PrimeConfig::cpu_count;
            saw_mem |= k.field == &PrimeConfig::memory_allowed_mb;
        }
    }
    const bool gpu_only = cfg.cpu_count == 0 && cfg.use_gpu != 0;
    if (!gpu_only && cfg.cpu_count <= 0) {
        cfg.cpu_count = cores_detected();
        saw_cpu = false;
    }
    if (cfg.memory_allowed_mb <= 0) {
        cfg.memory_allowed_mb = 10240;
        saw_mem = false;
    }
    if (!exists || !saw_cpu || !saw_mem) {
        std::ofstream out(path, std::ios::trunc);
        if (!out) fatal("Failed to write prime.ini at " + path);
        out << "CPU_count=" << cfg.cpu_count << "\nMemoryAllowed=" << cfg.memory_allowed_mb
            << "\nUseGPU=" << cfg.use_gpu << "\nGPU_device=" << cfg.gpu_device << "\n";
        info("Wrote prime.ini with CPU_count=" + std::to_string(cfg.cpu_count) +
             " MemoryAllowed=" + std::to_string(cfg.memory_allowed_mb) + " MB");
    }
    return cfg;
}

// ---------------------------------------------------------- worktodo.txt --

struct WorkItem {
    i128 b = 0, c = 0, P0 = 0, P0_original = 0, P1 = 0, N0 = 0, N1 = 0;
    uint64_t mod = 1, res = 0;
    uint64_t relations_restored = 0;

    bool in_class(i128 n) const {          // n % mod (truncating) == res (Types.hpp:28-31)
        return mod <= 1 || (uint64_t)(n % (i128)mod) == res;
    }
};

// The non-empty, trimmed ','-separated fields of s.
inline std::vector<std::string> fields(const std::string& s) {
    std::vector<std::string> out;
    size_t start = 0;
    for (;;) {
        const size_t comma = s.find(',', start);
        std::string f = strip(s.substr(start, comma == std::string::npos ? std::string::npos : comma - start));
        if (!f.empty()) out.push_back(std::move(f));
        if (comma == std::string::npos) break;
        start = comma + 1;
    }
    return out;
}

inline std::vector<WorkItem> read_worktodo(const std::string& path) {
    std::ifstream in(path);
    if (!in) fatal("Failed to open worktodo file: " + path);
    std::vector<WorkItem> items;
    size_t line_no = 0;
    for (std::string raw; std::getline(in, raw);) {
        ++line_no;
        std::string s = strip(raw);
        if (s.empty() || s[0] == '#') continue;
        if (s.compare(0, 7, "Factor=") == 0) s.erase(0, 7);
        const std::string where = "worktodo line " + std::to_string(line_no);
        const std::vector<std::string> f = fields(s);
        if (f.size() != 6 && f.size() != 8)
            fatal(where + " must have 6 or 8 comma-separated values (b,c,P0,P1,N0,N1[,mod,res])");
        WorkItem it;
        try {
            i128* const slot[6] = {&it.b, &it.c, &it.P0, &it.P1, &it.N0, &it.N1};
            for (int k = 0; k < 6; ++k) *slot[k] = i128_parse(f[k]);
            it.P0_original = it.P0;
            if (f.size() == 8) {
                it.mod = u64_reading(f[6]);
                it.res = u64_reading(f[7]);
                if (it.mod == 0 || it.res >= it.mod) throw std::invalid_argument("class must satisfy 0 <= res < mod");
            }
        } catch (const std::exception& ex) {
            fatal(where + " parse error: " + ex.what());
        }
        if (!(it.P0 < it.P1)) fatal(where + " requires P0 < P1");
        if (!(it.N0 < it.N1)) fatal(where + " requires N0 < N1");
        if (it.N1 - it.N0 > (i128)10000000) fatal(where + " range N1-N0 exceeds 10 million");
        items.push_back(it);
    }
    if (items.empty()) fatal("No work items found in " + path);
    return items;
}

// ------------------------------------------------------------ relations --

struct Relation {
    uint64_t p = 0, M = 0, q = 0;
};

inline std::string relation_text(const Relation& r) {
    char buf[80];
    const int n = std::snprintf(buf, sizeof(buf), "%llu, %llu, %llu\n", (unsigned long long)r.p,
                                (unsigned long long)r.M, (unsigned long long)r.q);
    return std::string(buf, (size_t)n);
}

// Stream-extraction style reader of one relations line.
class LineCursor {
public:
    explicit LineCursor(const std::string& s) : p_(s.c_str()) {}
    bool number(uint64_t* v) {                 // white space, optional sign, decimal digits
        while (is_space(*p_)) ++p_;
        const char* b = p_;
        bool neg = false;
        if (*p_ == '+' || *p_ == '-') neg = *p_++ == '-';
        if (!std::isdigit((unsigned char)*p_)) {
            p_ = b;
            return false;
        }
        u128 x = 0;
        while (std::isdigit((unsigned char)*p_)) {
            x = x * 10 + (unsigned)(*p_++ - '0');
            if (x > UINT64_MAX) return false;
        }
        *v = neg ? 0 - (uint64_t)x : (uint64_t)x;
        return true;
    }
    bool symbol(char want) {                   // white space, then exactly `want`
        while (is_space(*p_)) ++p_;
        if (*p_ != want) return false;
        ++p_;
        return true;
    }

private:
    const char* p_;
};

// The relation of one line; false if it does not start "p, M, q".
inline bool parse_relation(const std::string& line, Relation* r) {
    LineCursor cur(line);
    return cur.number(&r->p) && cur.symbol(',') && cur.number(&r->M) && cur.symbol(',') && cur.number(&r->q);
}

// The leading p of a line "p, ..."; false if the line does not start so.
inline bool leading_p(const std::string& line, uint64_t* p) {
    LineCursor cur(line);
    return cur.number(p) && cur.symbol(',');
}

inline std::vector<Relation> read_relations(const std::string& path) {
    std::vector<Relation> out;
    std::ifstream in(path);
    for (std::string line; std::getline(in, line);) {
        if (line.empty()) continue;
        Relation r;
        if (!parse_relation(line, &r)) fatal("Malformed relation line: " + line);
        out.push_back(r);
    }
    return out;
}

// ----------------------------------------------------------- candidates --

// Whether the reference's test finds b^n + c == p: the power is built one
// factor at a time and the test gives up once it exceeds 2p.
inline bool value_is_the_prime(const WorkItem& it, i128 n, uint64_t p) {
    const i128 bound = (i128)p * 2;
    if (it.b >= -1 && it.b <= 1) {                         // the power never exceeds 2p: b^n itself
        const i128 power = n <= 0 ? 1 : it.b == 0 ? 0 : (it.b == 1 || n % 2 == 0) ? 1 : -1;
        return power + it.c == (i128)p;
    }
    i128 power = 1;
    for (i128 e = 0; e < n; ++e) {
        power *= it.b;
        if (power > bound) return false;
    }
    return power + it.c == (i128)p;
}

// candidates[n - N0] = the relation primes dividing b^n + c, in relation order.
inline std::vector<std::vector<uint64_t>> candidate_primes(const WorkItem& it, const std::vector<Relation>& rel) {
    const i128 span = it.N1 - it.N0;
    std::vector<std::vector<uint64_t>> cand((size_t)span);
    for (const Relation& r : rel) {
        if (r.q == 0) continue;                            // no progression (never written by a siever)
        const i128 q = (i128)r.q;
        i128 off = ((i128)r.M - it.N0) % q;                // first n >= N0 with n == M (mod q)
        if (off < 0) off += q;
        for (i128 k = off; k < span; k += q) {
            if (value_is_the_prime(it, it.N0 + k, r.p)) continue;
            cand[(size_t)k].push_back(r.p);
        }
    }
    return cand;
}

// ---------------------------------------------------------- results.json --
//
// Output is produced as text directly: JsonText appends tokens with the
// separators a compact serialisation needs.  An existing results.json is
// copied into the new text token by token (Reserialiser): strings are
// decoded and re-escaped, integers re-printed from their value, other
// numbers kept as written, white space dropped.

inline void json_string(const std::string& s, std::string& out) {
    static const char hex[] = "0123456789abcdef";
    out += '"';
    for (unsigned char ch : s) {
        const char* esc = nullptr;
        switch (ch) {
            case '"': esc = "\\\""; break;
            case '\\': esc = "\\\\"; break;
            case '\b': esc = "\\b"; break;
            case '\f': esc = "\\f"; break;
            case '\n': esc = "\\n"; break;
            case '\r': esc = "\\r"; break;
            case '\t': esc = "\\t"; break;
            default: break;
        }
        if (esc) {
            out += esc;
        } else if (ch < 0x20) {
            out += "\\u00";
            out += hex[ch >> 4];
            out += hex[ch & 15];
        } else {
            out += (char)ch;
        }
    }
    out += '"';
}

// Integers beyond int64 are written as decimal strings (Results.hpp:59-70).
inline std::string json_number(i128 v) {
    const bool wide = v > (i128)INT64_MAX || v < (i128)INT64_MIN;
    std::string t = i128_text(v);
    return wide ? "\"" + t + "\"" : t;
}

class JsonText {
public:
    std::string out;
    void open(char bracket) {
        sep();
        out += bracket;
        fresh_ = true;
    }
    void close(char bracket) {
        out += bracket;
        fresh_ = false;
    }
    void key(const char* k) {
        sep();
        json_string(k, out);
        out += ':';
        fresh_ = true;
    }
    void raw(const std::string& token) {
        sep();
        out += token;
        fresh_ = false;
    }

private:
    void sep() {
        if (!fresh_ && !out.empty() && out.back() != ':') out += ',';
        fresh_ = false;
    }
    bool fresh_ = true;
};

class Reserialiser {
public:
    explicit Reserialiser(const std::string& text) : t_(text) {}

    // Re-serialises the whole text as one JSON value into out; throws on bad JSON.
    void value(std::string& out) {
        space();
        if (i_ >= t_.size()) fail("unexpected end of input");
        const char ch = t_[i_];
        if (ch == '[' || ch == '{') {
            const char end = ch == '[' ? ']' : '}';
            out += ch;
            ++i_;
            space();
            if (peek() == end) {
                ++i_;
                out += end;
                return;
            }
            for (bool first = true;; first = false) {
                if (!first) out += ',';
                if (end == '}') {
                    space();
                    if (peek() != '"') fail("expected an object key");
                    string(out);
                    space();
                    if (peek() != ':') fail("expected ':'");
                    ++i_;
                    out += ':';
                }
                value(out);
                space();
                const char c = peek();
                ++i_;
                if (c == end) break;
                if (c != ',') fail(end == ']' ? "expected ',' or ']'" : "expected ',' or '}'");
            }
            out += end;
        } else if (ch == '"') {
            string(out);
        } else if (ch == '-' || (ch >= '0' && ch <= '9')) {
            number(out);
        } else {
            for (const char* word : {"true", "false", "null"}) {
                const size_t n = std::strlen(word);
                if (t_.compare(i_, n, word) == 0) {
                    out += word;
                    i_ += n;
                    return;
                }
            }
            fail("unexpected character");
        }
    }
    bool at_end() {
        space();
        return i_ == t_.size();
    }
    bool starts_array() {
        space();
        return peek() == '[';
    }

private:
    [[noreturn]] void fail(const std::string& what) {
        throw std::runtime_error(what + " at offset " + std::to_string(i_));
    }
    char peek() const { return i_ < t_.size() ? t_[i_] : '\0'; }
    void space() {
        while (i_ < t_.size() && (t_[i_] == ' ' || t_[i_] == '\t' || t_[i_] == '\n' || t_[i_] == '\r')) ++i_;
    }
    unsigned hex4() {
        if (i_ + 4 > t_.size()) fail("short \\u escape");
        unsigned v = 0;
        for (int k = 0; k < 4; ++k) {
            const char c = t_[i_++];
            v <<= 4;
            if (c >= '0' && c <= '9') v |= (unsigned)(c - '0');
            else if (c >= 'a' && c <= 'f') v |= (unsigned)(c - 'a' + 10);
            else if (c >= 'A' && c <= 'F') v |= (unsigned)(c - 'A' + 10);
            else fail("bad \\u escape");
        }
        return v;
    }
    static void utf8(unsigned cp, std::string& s) {
        if (cp < 0x80) {
            s += (char)cp;
        } else if (cp < 0x800) {
            s += (char)(0xC0 | (cp >> 6));
            s += (char)(0x80 | (cp & 0x3F));
        } else if (cp < 0x10000) {
            s += (char)(0xE0 | (cp >> 12));
            s += (char)(0x80 | ((cp >> 6) & 0x3F));
            s += (char)(0x80 | (cp & 0x3F));
        } else {
            s += (char)(0xF0 | (cp >> 18));
            s += (char)(0x80 | ((cp >> 12) & 0x3F));
            s += (char)(0x80 | ((cp >> 6) & 0x3F));
            s += (char)(0x80 | (cp & 0x3F));
        }
    }
    void string(std::string& out) {
        ++i_;                                              // the opening quote
        std::string s;
        for (;;) {
            if (i_ >= t_.size()) fail("unterminated string");
            const char c = t_[i_++];
            if (c == '"') break;
            if ((unsigned char)c < 0x20) fail("control character in string");
            if (c != '\\') {
                s += c;
                continue;
            }
            if (i_ >= t_.size()) fail("unterminated escape");
            const char e = t_[i_++];
            const char* plain = std::strchr("\"\\/bfnrt", e);
            if (e != '\0' && plain) {
                static const char decoded[] = "\"\\/\b\f\n\r\t";
                s += decoded[plain - "\"\\/bfnrt"];
            } else if (e == 'u') {
                unsigned cp = hex4();
                if (cp >= 0xD800 && cp < 0xDC00 && t_.compare(i_, 2, "\\u") == 0) {
                    const size_t keep = i_;
                    i_ += 2;
                    const unsigned lo = hex4();
                    if (lo >= 0xDC00 && lo < 0xE000) cp = 0x10000 + ((cp - 0xD800) << 10) + (lo - 0xDC00);
                    else i_ = keep;
                }
                utf8(cp, s);
            } else {
                fail("bad escape");
            }
        }
        json_string(s, out);
    }
    void number(std::string& out) {
        const size_t b = i_;
        if (peek() == '-') ++i_;
        if (!std::isdigit((unsigned char)peek())) fail("bad number");
        if (peek() == '0' && i_ + 1 < t_.size() && std::isdigit((unsigned char)t_[i_ + 1])) fail("leading zero");
        while (std::isdigit((unsigned char)peek())) ++i_;
        bool integral = true;
        if (peek() == '.') {
            integral = false;
            ++i_;
            if (!std::isdigit((unsigned char)peek())) fail("bad fraction");
            while (std::isdigit((unsigned char)peek())) ++i_;
        }
        if (peek() == 'e' || peek() == 'E') {
            integral = false;
            ++i_;
            if (peek() == '+' || peek() == '-') ++i_;
            if (!std::isdigit((unsigned char)peek())) fail("bad exponent");
            while (std::isdigit((unsigned char)peek())) ++i_;
        }
        const std::string tok = t_.substr(b, i_ - b);
        if (integral && tok.size() <= 21) {
            const i128 v = i128_parse(tok[0] == '-' ? "-" + strip_zeros(tok.substr(1)) : strip_zeros(tok));
            if (v >= (i128)INT64_MIN && v <= (i128)UINT64_MAX) {
                out += i128_text(v);
                return;
            }
        }
        out += tok;
    }
    static std::string strip_zeros(const std::string& d) {     // decimal digits without an octal reading
        size_t k = 0;
        while (k + 1 < d.size() && d[k] == '0') ++k;
        return d.substr(k);
    }

    const std::string& t_;
    size_t i_ = 0;
};

// The entry of one finished item (Results.hpp:72-110).
inline std::string results_entry(const WorkItem& it, const std::vector<std::vector<uint64_t>>& cand,
                                 const std::string& timestamp) {
    JsonText j;
    j.open('{');
    j.key("Timestamp");
    std::string ts;
    json_string(timestamp, ts);
    j.raw(ts);
    const std::pair<const char*, i128> head[] = {{"b", it.b},   {"c", it.c},   {"P0", it.P0_original},
                                                 {"P1", it.P1}, {"N0", it.N0}, {"N1", it.N1}};
    for (const auto& [name, v] : head) {
        j.key(name);
        j.raw(json_number(v));
    }
    j.key("prp");
    j.open('[');
    for (size_t k = 0; k < cand.size(); ++k) {
        const i128 n = it.N0 + (i128)k;
        if (it.in_class(n) && cand[k].empty()) j.raw(json_number(n));
    }
    j.close(']');
    j.key("factored");
    j.open('[');
    for (size_t k = 0; k < cand.size(); ++k) {
        const i128 n = it.N0 + (i128)k;
        if (!it.in_class(n) || cand[k].empty()) continue;
        j.open('{');
        j.key("n");
        j.raw(json_number(n));
        j.key("factors");
        j.open('[');
        for (uint64_t p : cand[k]) j.raw(json_number((i128)p));
        j.close(']');
        j.close('}');
    }
    j.close(']');
    j.close('}');
    return j.out;
}

// Appends an entry to the results file: the file's array re-serialised, then the entry.
inline void append_result(const std::string& path, const std::string& entry) {
    std::string text;
    {
        std::ifstream in(path, std::ios::binary);
        if (in) text.assign(std::istreambuf_iterator<char>(in), std::istreambuf_iterator<char>());
    }
    std::string out;
    if (text.empty()) {
        out = "[" + entry + "]";
    } else {
        try {
            Reserialiser rs(text);
            if (!rs.starts_array()) {
                std::string probe;
                rs.value(probe);                           // a malformed file is a parse error first
                if (!rs.at_end()) throw std::runtime_error("extra data after the JSON value");
                fatal("results.json must contain a JSON array");
            }
            rs.value(out);
            if (!rs.at_end()) throw std::runtime_error("extra data after the JSON value");
        } catch (const std::exception& ex) {
            fatal(std::string("Failed to parse results.json: ") + ex.what());
        }
        out.insert(out.size() - 1, (out.size() > 2 ? "," : "") + entry);
    }
    std::ofstream f(path, std::ios::trunc | std::ios::binary);
    if (!f) fatal("Failed to write results.json");
    f << out << '\n';
    f.flush();
    if (!f) fatal("Failed while saving results.json");
}

// ------------------------------------------------------------ reporting --

inline std::string hms(double seconds) {                    // Results.hpp:16-25
    const long long t = (long long)seconds;
    char buf[48];
    std::snprintf(buf, sizeof(buf), "%lld:%02lld:%02lld", t / 3600, t % 3600 / 60, t % 60);
    return buf;
}

inline std::string final_status(const WorkItem& it, const std::vector<std::vector<uint64_t>>& cand, double secs) {
    size_t total = 0, alive = 0;
    for (size_t k = 0; k < cand.size(); ++k) {
        if (!it.in_class(it.N0 + (i128)k)) continue;
        ++total;
        alive += cand[k].empty() ? 1 : 0;
    }
    char buf[200];
    std::snprintf(buf, sizeof(buf), "Final status: %zu/%zu candidates survived (%.2f%% survival rate), elapsed %s",
                  alive, total, total ? 100.0 * (double)alive / (double)total : 0.0, hms(secs).c_str());
    return buf;
}

}  // namespace mpsio
