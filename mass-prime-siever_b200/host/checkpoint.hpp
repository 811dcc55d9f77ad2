// checkpoint.hpp -- resumable progress over core_<id>.p relation files.
//
// Specification (the reference's resume rule, Worker.hpp:369-463, and its
// merge, Worker.hpp:469-495):
//  * A run appends each finished chunk's relations to core_<id>.p.  Every
//    core file's last relation line therefore carries the largest p of a
//    chunk whose relations are complete, so the smallest such p over all
//    core files is a point below which every p has been sieved.
//  * On start, if any core file ends in a relation line, the resume point R
//    is that smallest p.  R <= P0 keeps P0 ("Checkpoint not ahead of current
//    P0, starting from original P0."); no such file keeps P0 ("No
//    checkpoint found, starting from original P0.").  Otherwise P0 = R,
//    every core file keeps only its relation lines with p < R (blank and
//    unreadable lines are dropped), and the log says "Checkpoint recovered:
//    new P0 = R, relations restored = <lines kept>".
//  * This worker also writes core_progress.txt after each chunk: one line
//    "<b> <c> <P0> <P1> <N0> <N1> <mod> <res> <p_done>" (P0 the item's
//    original P0).  When it names the item being resumed, p_done replaces R
//    (it is exact even when the last chunk found no relation).
//  * The merge writes every relation line of the core files into relations.p
//    in increasing p and deletes the core files.
//
// Core files are looked for at ids 0 .. kCoreIds - 1 (the reference stops at
// the first two missing ids in a row; looking at all ids also finds the
// files of a run whose first workers wrote nothing).
#pragma once

#include "formats.hpp"

#include <algorithm>
#include <cstdio>
#include <fcntl.h>
#include <unistd.h>

namespace mpsio {

constexpr int kCoreIds = 1024;
inline const char* kProgressFile = "core_progress.txt";

inline std::string core_file(int id) { return "core_" + std::to_string(id) + ".p"; }

struct CoreFile {
    int id;
    std::vector<std::pair<uint64_t, std::string>> lines;   // relation lines with their p, file order
    bool last_is_relation = false;                         // the file's last non-blank line is one
    uint64_t last_p = 0;
};

inline std::vector<CoreFile> scan_core_files() {
    std::vector<CoreFile> files;
    for (int id = 0; id < kCoreIds; ++id) {
        std::ifstream in(core_file(id));
        if (!in) continue;
        CoreFile cf{id, {}, false, 0};
        for (std::string line; std::getline(in, line);) {
            if (line.empty()) continue;
            uint64_t p = 0;
            cf.last_is_relation = leading_p(line, &p);
            if (cf.last_is_relation) {
                cf.last_p = p;
                cf.lines.emplace_back(p, line);
            }
        }
        files.push_back(std::move(cf));
    }
    return files;
}

// Writes `text` to `path` through a temporary file and a rename.
inline bool replace_file(const std::string& path, const std::string& text) {
    const std::string tmp = path + ".tmp";
    {
        std::ofstream out(tmp, std::ios::trunc | std::ios::binary);
        if (!out) return false;
        out << text;
        out.flush();
        if (!out) return false;
    }
    return std::rename(tmp.c_str(), path.c_str()) == 0;
}

inline std::string progress_line(const WorkItem& it) {
    return i128_text(it.b) + ' ' + i128_text(it.c) + ' ' + i128_text(it.P0_original) + ' ' + i128_text(it.P1) + ' ' +
           i128_text(it.N0) + ' ' + i128_text(it.N1) + ' ' + std::to_string(it.mod) + ' ' + std::to_string(it.res);
}

// The exact progress of this item, if the progress file names it.
inline bool read_progress(const WorkItem& it, i128* p_done) {
    std::ifstream in(kProgressFile);
    std::string line;
    if (!in || !std::getline(in, line)) return false;
    const std::string head = progress_line(it) + ' ';
    if (line.size() <= head.size() || line.compare(0, head.size(), head) != 0) return false;
    try {
        *p_done = i128_parse(strip(line.substr(head.size())));
    } catch (const std::exception&) {
        return false;
    }
    return *p_done >= it.P0_original && *p_done <= it.P1;
}

// Records that every p below p_done is sieved (atomic replace).
inline void write_progress(const WorkItem& it, i128 p_done) {
    if (!replace_file(kProgressFile, progress_line(it) + ' ' + i128_text(p_done) + '\n'))
        fatal(std::string("Failed to replace ") + kProgressFile);
}

// Moves it.P0 to the resume point and trims the core files to it.
inline void resume(WorkItem& it) {
    std::vector<CoreFile> files = scan_core_files();
    bool found = false;
    i128 R = it.P1;
    for (const CoreFile& cf : files)
        if (cf.last_is_relation && (i128)cf.last_p < R) {
            R = (i128)cf.last_p;
            found = true;
        }
    i128 exact = 0;
    if (read_progress(it, &exact) && exact > it.P0) {
        R = exact;
        found = true;
    }
    if (!found) {
        info("No checkpoint found, starting from original P0.");
        return;
    }
    if (R <= it.P0) {
        info("Checkpoint not ahead of current P0, starting from original P0.");
        return;
    }
    uint64_t kept = 0;
    for (const CoreFile& cf : files) {
        std::string text;
        for (const auto& [p, line] : cf.lines)
            if ((i128)p < R) {
                text += line;
                text += '\n';
                ++kept;
            }
        if (!replace_file(core_file(cf.id), text)) fatal("Failed to trim checkpoint file: " + core_file(cf.id));
    }
    it.P0 = R;
    it.relations_restored = kept;
    info("Checkpoint recovered: new P0 = " + i128_text(R) + ", relations restored = " + std::to_string(kept));
}

// Appends relation lines to core_<id>.p and makes them durable before the
// caller records the chunk as done.
inline void append_core(int id, const std::vector<Relation>& rel) {
    if (rel.empty()) return;
    const std::string path = core_file(id);
    std::string text;
    for (const Relation& r : rel) text += relation_text(r);
    const int fd = ::open(path.c_str(), O_WRONLY | O_CREAT | O_APPEND, 0644);
    if (fd < 0) fatal("Failed to append to " + path);
    size_t done = 0;
    while (done < text.size()) {
        const ssize_t w = ::write(fd, text.data() + done, text.size() - done);
        if (w <= 0) {
            ::close(fd);
            fatal("Failed to append to " + path);
        }
        done += (size_t)w;
    }
    if (::fsync(fd) != 0 || ::close(fd) != 0) fatal("Failed to flush " + path);
}

// All relation lines of the core files, in increasing p, into relations.p;
// the core files are removed.
inline void merge_core_files() {
    std::vector<std::pair<uint64_t, std::string>> all;
    std::vector<int> ids;
    for (CoreFile& cf : scan_core_files()) {
        ids.push_back(cf.id);
        for (auto& pl : cf.lines) all.push_back(std::move(pl));
    }
    std::stable_sort(all.begin(), all.end(), [](const auto& a, const auto& b) { return a.first < b.first; });
    std::ofstream out("relations.p", std::ios::binary | std::ios::trunc);
    if (!out) fatal("Failed to create relations.p");
    for (const auto& pl : all) out << pl.second << '\n';
    out.flush();
    if (!out) fatal("Failed while writing relations.p");
    out.close();
    for (int id : ids) std::remove(core_file(id).c_str());
}

}  // namespace mpsio
