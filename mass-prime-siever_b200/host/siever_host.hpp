// siever_host.hpp -- the reference's host surface around the GPU path.
//
// prime.ini and worktodo.txt parsing (Config.hpp:50-200), the logger line
// format (Logger.hpp:15-29, 143-155), checkpoint/resume over core_<id>.p
// files (Worker.hpp:369-495), relations.p parsing and application to the
// candidate exponents (Worker.hpp:497-559), and the results.json entry
// (Results.hpp:57-140), restated for a GPU-only worker that calls
// libmps_b200.so.  Output formats are byte-compatible with the reference.
#pragma once

#include <algorithm>
#include <cctype>
#include <chrono>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <ctime>
#include <fstream>
#include <iostream>
#include <mutex>
#include <sstream>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

namespace mpsh {

typedef __int128 i128;
typedef unsigned __int128 u128;

// ---------------------------------------------------------------- logging --

// "YYYY-MM-DD HH:MM:SS UTC+0" (Logger.hpp:15-29).
inline std::string utc_timestamp(std::time_t t) {
    std::tm tm{};
    gmtime_r(&t, &tm);
    char buf[64];
    std::snprintf(buf, sizeof(buf), "%04d-%02d-%02d %02d:%02d:%02d UTC+0", tm.tm_year + 1900, tm.tm_mon + 1,
                  tm.tm_mday, tm.tm_hour, tm.tm_min, tm.tm_sec);
    return buf;
}
inline std::string now_timestamp() { return utc_timestamp(std::time(nullptr)); }

class Logger {
public:
    static Logger& instance() {
        static Logger log;
        return log;
    }
    void init(const std::string& path) {
        std::lock_guard<std::mutex> g(mu_);
        if (file_.is_open()) return;
        file_.open(path, std::ios::app);
        if (!file_) throw std::runtime_error("Failed to open log file: " + path);
    }
    void write(const char* level, const std::string& msg) {
        std::lock_guard<std::mutex> g(mu_);
        const std::string line = now_timestamp() + " [" + level + "] " + msg;
        std::cerr << line << std::endl;
        if (file_.is_open()) {
            file_ << line << std::endl;
            file_.flush();
        }
    }

private:
    std::mutex mu_;
    std::ofstream file_;
};

inline void log_info(const std::string& m) { Logger::instance().write("INFO", m); }
[[noreturn]] inline void log_fatal(const std::string& m) {
    Logger::instance().write("FATAL", m);
    std::exit(1);
}

// ---------------------------------------------------------------- numbers --

inline std::string to_string128(i128 v) {
    const bool neg = v < 0;
    u128 u = neg ? (u128)0 - (u128)v : (u128)v;
    std::string s;
    do {
        s.insert(s.begin(), char('0' + int(u % 10)));
        u /= 10;
    } while (u);
    if (neg) s.insert(s.begin(), '-');
    return s;
}

// Decimal text -> 128-bit integer (boost int128_t's string constructor:
// optional sign, decimal digits; anything else is an error).
inline i128 parse128(const std::string& s) {
    size_t i = 0;
    bool neg = false;
    if (i < s.size() && (s[i] == '-' || s[i] == '+')) neg = s[i++] == '-';
    if (i >= s.size()) throw std::invalid_argument("empty number");
    u128 v = 0;
    for (; i < s.size(); ++i) {
        if (!std::isdigit((unsigned char)s[i])) throw std::invalid_argument("not a decimal integer: " + s);
        const u128 nv = v * 10 + (u128)(s[i] - '0');
        if (nv / 10 != v || nv > ((u128)1 << 127)) throw std::out_of_range("integer out of 128-bit range: " + s);
        v = nv;
    }
    if (!neg && v == ((u128)1 << 127)) throw std::out_of_range("integer out of 128-bit range: " + s);
    return neg ? (i128)((u128)0 - v) : (i128)v;
}

inline std::string trim(std::string v) {
    const auto ns = [](unsigned char ch) { return !std::isspace(ch); };
    v.erase(v.begin(), std::find_if(v.begin(), v.end(), ns));
    v.erase(std::find_if(v.rbegin(), v.rend(), ns).base(), v.end());
    return v;
}

// ----------------------------------------------------------------- config --

struct PrimeConfig {                 // Config.hpp:16-26
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

inline int detect_cpu_count() {
    const int hw = (int)std::thread::hardware_concurrency();
    return hw > 0 ? hw : 1;
}

// Config.hpp:50-122, including its rewrite of prime.ini (4 keys) when
// CPU_count or MemoryAllowed is missing or the file does not exist.
inline PrimeConfig load_prime_config(const std::string& path) {
    PrimeConfig c;
    c.cpu_count = detect_cpu_count();
    std::ifstream in(path);
    bool has_cpu = false, has_mem = false;
    if (in) {
        std::string line;
        while (std::getline(in, line)) {
            line = trim(line);
            if (line.empty() || line[0] == '#') continue;
            const auto pos = line.find('=');
            if (pos == std::string::npos) continue;
            const std::string key = trim(line.substr(0, pos)), value = trim(line.substr(pos + 1));
            if (key.empty()) continue;
            if (key == "CPU_count") {
                c.cpu_count = std::stoi(value);
                has_cpu = true;
            } else if (key == "UseGPU") {
                c.use_gpu = std::stoi(value);
            } else if (key == "GPU_device") {
                c.gpu_device = std::stoi(value);
            } else if (key == "GPU_backend") {
                c.gpu_backend = value;
            } else if (key == "GPU_threads") {
                c.gpu_threads = std::max(1, std::stoi(value));
            } else if (key == "GPU_sieve") {
                c.gpu_sieve = std::stoi(value);
            } else if (key == "GPU_classes") {
                c.gpu_classes = std::stoi(value);
            } else if (key == "GPU_strict") {
                c.gpu_strict = std::stoi(value);
            } else if (key == "MemoryAllowed") {
                c.memory_allowed_mb = std::stoi(value);
                has_mem = true;
            }
        }
    }
    if (c.cpu_count == 0 && c.use_gpu != 0) {
    } else if (c.cpu_count <= 0) {
        c.cpu_count = detect_cpu_count();
        has_cpu = false;
    }
    if (c.memory_allowed_mb <= 0) {
        c.memory_allowed_mb = 10240;
        has_mem = false;
    }
    const bool existed = (bool)std::ifstream(path);
    if (!has_cpu || !has_mem || !existed) {
        std::ofstream out(path, std::ios::trunc);
        if (!out) log_fatal("Failed to write prime.ini at " + path);
        out << "CPU_count=" << c.cpu_count << "\n";
        out << "MemoryAllowed=" << c.memory_allowed_mb << "\n";
        out << "UseGPU=" << c.use_gpu << "\n";
        out << "GPU_device=" << c.gpu_device << "\n";
        log_info("Wrote prime.ini with CPU_count=" + std::to_string(c.cpu_count) +
                 " MemoryAllowed=" + std::to_string(c.memory_allowed_mb) + " MB");
    }
    return c;
}

struct WorkItem {                    // Types.hpp:14-26
    i128 b = 0, c = 0, P0 = 0, P0_original = 0, P1 = 0, N0 = 0, N1 = 0;
    uint64_t relations_restored = 0;
    uint64_t cls_mod = 1, cls_res = 0;
};

inline bool in_class(const WorkItem& it, i128 n) {       // Types.hpp:28-31
    if (it.cls_mod <= 1) return true;
    return (uint64_t)(n % (i128)it.cls_mod) == it.cls_res;
}

// Config.hpp:124-200.  Errors end the program with the reference's messages.
inline std::vector<WorkItem> load_worktodo(const std::string& path) {
    std::ifstream in(path);
    if (!in) log_fatal("Failed to open worktodo file: " + path);
    std::vector<WorkItem> items;
    std::string line;
    size_t line_no = 0;
    while (std::getline(in, line)) {
        ++line_no;
        line = trim(line);
        if (line.empty() || line[0] == '#') continue;
        const std::string prefix = "Factor=";
        if (line.rfind(prefix, 0) == 0) line = line.substr(prefix.size());
        std::vector<std::string> parts;
        std::stringstream ss(line);
        std::string tok;
        while (std::getline(ss, tok, ',')) {
            tok = trim(tok);
            if (!tok.empty()) parts.push_back(tok);
        }
        if (parts.size() != 6 && parts.size() != 8)
            log_fatal("worktodo line " + std::to_string(line_no) +
                      " must have 6 or 8 comma-separated values (b,c,P0,P1,N0,N1[,mod,res])");
        WorkItem it;
        try {
            it.b = parse128(parts[0]);
            it.c = parse128(parts[1]);
            it.P0 = parse128(parts[2]);
            it.P0_original = it.P0;
            it.P1 = parse128(parts[3]);
            it.N0 = parse128(parts[4]);
            it.N1 = parse128(parts[5]);
            if (parts.size() == 8) {
                it.cls_mod = std::stoull(parts[6]);
                it.cls_res = std::stoull(parts[7]);
                if (it.cls_mod == 0 || it.cls_res >= it.cls_mod)
                    throw std::invalid_argument("class must satisfy 0 <= res < mod");
            }
        } catch (const std::exception& ex) {
            log_fatal("worktodo line " + std::to_string(line_no) + " parse error: " + ex.what());
        }
        if (it.P0 >= it.P1) log_fatal("worktodo line " + std::to_string(line_no) + " requires P0 < P1");
        if (it.N0 >= it.N1) log_fatal("worktodo line " + std::to_string(line_no) + " requires N0 < N1");
        if (it.N1 - it.N0 > (i128)10000000)
            log_fatal("worktodo line " + std::to_string(line_no) + " range N1-N0 exceeds 10 million");
        items.push_back(it);
    }
    if (items.empty()) log_fatal("No work items found in " + path);
    return items;
}

// -------------------------------------------------------------- relations --

struct Relation {
    uint64_t p = 0, M = 0, q = 0;
};

inline std::string relation_line(const Relation& r) {   // Worker.hpp:294-297
    char buf[96];
    std::snprintf(buf, sizeof(buf), "%llu, %llu, %llu\n", (unsigned long long)r.p, (unsigned long long)r.M,
                  (unsigned long long)r.q);
    return buf;
}

// Worker.hpp:497-525
inline std::vector<Relation> load_relations(const std::string& path) {
    std::ifstream in(path);
    std::vector<Relation> out;
    if (!in) return out;
    std::string line;
    while (std::getline(in, line)) {
        if (line.empty()) continue;
        std::stringstream ps(line);
        char comma = 0;
        unsigned long long p = 0, M = 0, q = 0;
        if (!(ps >> p) || !(ps >> comma) || comma != ',' || !(ps >> M) || !(ps >> comma) || comma != ',' ||
            !(ps >> q))
            log_fatal("Malformed relation line: " + line);
        out.push_back(Relation{p, M, q});
    }
    return out;
}

inline i128 ceil_div(i128 a, i128 b) { return a >= 0 ? (a + b - 1) / b : a / b; }    // Math.hpp:176-184
inline i128 floor_div(i128 a, i128 b) { return a >= 0 ? a / b : (a - b + 1) / b; }   // Math.hpp:186-194

// Worker.hpp:527-559: candidates[n - N0] = the primes dividing b^n + c, in
// relation order, skipping b^n + c == p itself.
inline std::vector<std::vector<uint64_t>> apply_relations(const WorkItem& it, const std::vector<Relation>& rel) {
    const size_t count = (size_t)(it.N1 - it.N0);
    std::vector<std::vector<uint64_t>> cand(count);
    for (const Relation& r : rel) {
        const i128 q = (i128)r.q, M = (i128)r.M;
        const i128 x0 = ceil_div(it.N0 - M, q), x1 = floor_div(it.N1 - 1 - M, q);
        for (i128 x = x0; x <= x1; ++x) {
            const i128 n = q * x + M;
            const i128 index = n - it.N0;
            if (index < 0 || index >= (i128)count) continue;
            i128 value = 1;
            bool fits = true;
            for (i128 e = 0; e < n && fits; ++e) {
                value *= it.b;
                if (value > (i128)r.p * 2) fits = false;
            }
            if (fits && value + it.c == (i128)r.p) continue;
            cand[(size_t)index].push_back(r.p);
        }
    }
    return cand;
}

// ------------------------------------------------------------ results.json --
//
// A small JSON reader/writer for the subset results.json uses (arrays,
// objects, strings, integers, true/false/null).  serialize() writes what
// boost::json::serialize writes for these values: no whitespace, object
// keys in insertion order, strings escaped as boost escapes them.  A
// non-integer number (never written by either program) is kept as the text
// it was read from; boost would re-format it.

struct JValue {
    enum Kind { Null, Bool, Int, UInt, Raw, Str, Arr, Obj } kind = Null;
    bool b = false;
    int64_t i = 0;
    uint64_t u = 0;
    std::string s;
    std::vector<JValue> arr;
    std::vector<std::pair<std::string, JValue>> obj;
};

inline void json_escape(const std::string& s, std::string& out) {
    out += '"';
    for (unsigned char ch : s) {
        switch (ch) {
            case '"': out += "\\\""; break;
            case '\\': out += "\\\\"; break;
            case '\b': out += "\\b"; break;
            case '\f': out += "\\f"; break;
            case '\n': out += "\\n"; break;
            case '\r': out += "\\r"; break;
            case '\t': out += "\\t"; break;
            default:
                if (ch < 0x20) {
                    char buf[8];
                    std::snprintf(buf, sizeof(buf), "\\u%04x", ch);
                    out += buf;
                } else {
                    out += (char)ch;
                }
        }
    }
    out += '"';
}

inline void serialize(const JValue& v, std::string& out) {
    switch (v.kind) {
        case JValue::Null: out += "null"; break;
        case JValue::Bool: out += v.b ? "true" : "false"; break;
        case JValue::Int: out += std::to_string(v.i); break;
        case JValue::UInt: out += std::to_string(v.u); break;
        case JValue::Raw: out += v.s; break;
        case JValue::Str: json_escape(v.s, out); break;
        case JValue::Arr:
            out += '[';
            for (size_t k = 0; k < v.arr.size(); ++k) {
                if (k) out += ',';
                serialize(v.arr[k], out);
            }
            out += ']';
            break;
        case JValue::Obj:
            out += '{';
            for (size_t k = 0; k < v.obj.size(); ++k) {
                if (k) out += ',';
                json_escape(v.obj[k].first, out);
                out += ':';
                serialize(v.obj[k].second, out);
            }
            out += '}';
            break;
    }
}

struct JParser {
    const std::string& t;
    size_t i = 0;
    explicit JParser(const std::string& text) : t(text) {}
    void ws() {
        while (i < t.size() && (t[i] == ' ' || t[i] == '\n' || t[i] == '\r' || t[i] == '\t')) ++i;
    }
    [[noreturn]] void err(const std::string& m) { throw std::runtime_error(m + " at offset " + std::to_string(i)); }
    JValue value() {
        ws();
        if (i >= t.size()) err("unexpected end");
        const char ch = t[i];
        JValue v;
        if (ch == '[') {
            v.kind = JValue::Arr;
            ++i;
            ws();
            if (i < t.size() && t[i] == ']') {
                ++i;
                return v;
            }
            for (;;) {
                v.arr.push_back(value());
                ws();
                if (i < t.size() && t[i] == ',') {
                    ++i;
                    continue;
                }
                if (i < t.size() && t[i] == ']') {
                    ++i;
                    return v;
                }
                err("expected , or ]");
            }
        }
        if (ch == '{') {
            v.kind = JValue::Obj;
            ++i;
            ws();
            if (i < t.size() && t[i] == '}') {
                ++i;
                return v;
            }
            for (;;) {
                ws();
                JValue k = value();
                if (k.kind != JValue::Str) err("object key must be a string");
                ws();
                if (i >= t.size() || t[i] != ':') err("expected :");
                ++i;
                v.obj.push_back({k.s, value()});
                ws();
                if (i < t.size() && t[i] == ',') {
                    ++i;
                    continue;
                }
                if (i < t.size() && t[i] == '}') {
                    ++i;
                    return v;
                }
                err("expected , or }");
            }
        }
        if (ch == '"') {
            v.kind = JValue::Str;
            ++i;
            while (i < t.size() && t[i] != '"') {
                if (t[i] == '\\') {
                    ++i;
                    if (i >= t.size()) err("bad escape");
                    const char e = t[i++];
                    switch (e) {
                        case '"': v.s += '"'; break;
                        case '\\': v.s += '\\'; break;
                        case '/': v.s += '/'; break;
                        case 'b': v.s += '\b'; break;
                        case 'f': v.s += '\f'; break;
                        case 'n': v.s += '\n'; break;
                        case 'r': v.s += '\r'; break;
                        case 't': v.s += '\t'; break;
                        case 'u': {
                            if (i + 4 > t.size()) err("bad \\u escape");
                            unsigned cp = (unsigned)std::stoul(t.substr(i, 4), nullptr, 16);
                            i += 4;
                            if (cp >= 0xD800 && cp < 0xDC00 && i + 6 <= t.size() && t[i] == '\\' && t[i + 1] == 'u') {
                                const unsigned lo = (unsigned)std::stoul(t.substr(i + 2, 4), nullptr, 16);
                                if (lo >= 0xDC00 && lo < 0xE000) {
                                    cp = 0x10000 + ((cp - 0xD800) << 10) + (lo - 0xDC00);
                                    i += 6;
                                }
                            }
                            if (cp < 0x80) v.s += (char)cp;
                            else if (cp < 0x800) {
                                v.s += (char)(0xC0 | (cp >> 6));
                                v.s += (char)(0x80 | (cp & 0x3F));
                            } else if (cp < 0x10000) {
                                v.s += (char)(0xE0 | (cp >> 12));
                                v.s += (char)(0x80 | ((cp >> 6) & 0x3F));
                                v.s += (char)(0x80 | (cp & 0x3F));
                            } else {
                                v.s += (char)(0xF0 | (cp >> 18));
                                v.s += (char)(0x80 | ((cp >> 12) & 0x3F));
                                v.s += (char)(0x80 | ((cp >> 6) & 0x3F));
                                v.s += (char)(0x80 | (cp & 0x3F));
                            }
                            break;
                        }
                        default: err("bad escape");
                    }
                } else {
                    v.s += t[i++];
                }
            }
            if (i >= t.size()) err("unterminated string");
            ++i;
            return v;
        }
        if (t.compare(i, 4, "true") == 0) {
            i += 4;
            v.kind = JValue::Bool;
            v.b = true;
            return v;
        }
        if (t.compare(i, 5, "false") == 0) {
            i += 5;
            v.kind = JValue::Bool;
            return v;
        }
        if (t.compare(i, 4, "null") == 0) {
            i += 4;
            return v;
        }
        if (ch == '-' || std::isdigit((unsigned char)ch)) {
            size_t j = i + (ch == '-' ? 1 : 0);
            while (j < t.size() && std::isdigit((unsigned char)t[j])) ++j;
            if (j < t.size() && (t[j] == '.' || t[j] == 'e' || t[j] == 'E')) {
                while (j < t.size() && (std::isdigit((unsigned char)t[j]) || t[j] == '.' || t[j] == 'e' ||
                                        t[j] == 'E' || t[j] == '+' || t[j] == '-'))
                    ++j;
                v.kind = JValue::Raw;
                v.s = t.substr(i, j - i);
                i = j;
                return v;
            }
            const std::string num = t.substr(i, j - i);
            i = j;
            const i128 x = parse128(num);
            if (x >= INT64_MIN && x <= INT64_MAX) {
                v.kind = JValue::Int;
                v.i = (int64_t)x;
            } else if (x >= 0 && x <= (i128)UINT64_MAX) {
                v.kind = JValue::UInt;
                v.u = (uint64_t)x;
            } else {
                err("integer out of range");
            }
            return v;
        }
        err("unexpected character");
    }
};

// Results.hpp:59-70: an integer, or its decimal string beyond int64.
inline JValue json_int(i128 x) {
    JValue v;
    if (x > (i128)INT64_MAX || x < (i128)INT64_MIN) {
        v.kind = JValue::Str;
        v.s = to_string128(x);
    } else {
        v.kind = JValue::Int;
        v.i = (int64_t)x;
    }
    return v;
}
inline JValue json_uint(uint64_t x) {
    JValue v;
    if (x > (uint64_t)INT64_MAX) {
        v.kind = JValue::Str;
        v.s = std::to_string(x);
    } else {
        v.kind = JValue::Int;
        v.i = (int64_t)x;
    }
    return v;
}

// Results.hpp:72-110: the entry of one finished item.
inline JValue results_entry(const WorkItem& it, const std::vector<std::vector<uint64_t>>& cand,
                            const std::string& timestamp) {
    JValue e;
    e.kind = JValue::Obj;
    JValue ts;
    ts.kind = JValue::Str;
    ts.s = timestamp;
    e.obj.push_back({"Timestamp", ts});
    e.obj.push_back({"b", json_int(it.b)});
    e.obj.push_back({"c", json_int(it.c)});
    e.obj.push_back({"P0", json_int(it.P0_original)});
    e.obj.push_back({"P1", json_int(it.P1)});
    e.obj.push_back({"N0", json_int(it.N0)});
    e.obj.push_back({"N1", json_int(it.N1)});
    JValue prp, factored;
    prp.kind = factored.kind = JValue::Arr;
    for (size_t k = 0; k < cand.size(); ++k) {
        const i128 n = it.N0 + (i128)k;
        if (!in_class(it, n)) continue;
        if (cand[k].empty()) {
            prp.arr.push_back(json_int(n));
            continue;
        }
        JValue fe, fs;
        fe.kind = JValue::Obj;
        fs.kind = JValue::Arr;
        fe.obj.push_back({"n", json_int(n)});
        for (uint64_t f : cand[k]) fs.arr.push_back(json_uint(f));
        fe.obj.push_back({"factors", fs});
        factored.arr.push_back(fe);
    }
    e.obj.push_back({"prp", prp});
    e.obj.push_back({"factored", factored});
    return e;
}

// Results.hpp:111-140: parse results.json (if any), append, rewrite.
inline void append_results_json(const std::string& path, const JValue& entry) {
    JValue all;
    all.kind = JValue::Arr;
    {
        std::ifstream in(path);
        if (in) {
            const std::string content((std::istreambuf_iterator<char>(in)), std::istreambuf_iterator<char>());
            if (!content.empty()) {
                try {
                    JParser ps(content);
                    JValue parsed = ps.value();
                    ps.ws();
                    if (ps.i != content.size()) throw std::runtime_error("trailing characters");
                    if (parsed.kind != JValue::Arr) log_fatal("results.json must contain a JSON array");
                    all = std::move(parsed);
                } catch (const std::exception& ex) {
                    log_fatal(std::string("Failed to parse results.json: ") + ex.what());
                }
            }
        }
    }
    all.arr.push_back(entry);
    std::string text;
    serialize(all, text);
    std::ofstream out(path, std::ios::trunc);
    if (!out) log_fatal("Failed to write results.json");
    out << text << '\n';
    out.flush();
    if (!out) log_fatal("Failed while saving results.json");
}

// Results.hpp:16-55
inline std::string format_elapsed(double seconds) {
    const long long t = (long long)seconds;
    char buf[64];
    std::snprintf(buf, sizeof(buf), "%lld:%02lld:%02lld", t / 3600, (t % 3600) / 60, t % 60);
    return buf;
}

inline std::string final_status(const WorkItem& it, const std::vector<std::vector<uint64_t>>& cand, double elapsed) {
    size_t total = 0, surv = 0;
    for (size_t k = 0; k < cand.size(); ++k) {
        if (!in_class(it, it.N0 + (i128)k)) continue;
        ++total;
        if (cand[k].empty()) ++surv;
    }
    const double rate = total == 0 ? 0.0 : 100.0 * (double)surv / (double)total;
    char buf[256];
    std::snprintf(buf, sizeof(buf), "Final status: %zu/%zu candidates survived (%.2f%% survival rate), elapsed %s",
                  surv, total, rate, format_elapsed(elapsed).c_str());
    return buf;
}

}  // namespace mpsh
