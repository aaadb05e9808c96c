// cnm_snapshot_text.hpp -- text of a state snapshot, formatted on several threads.
//
// A snapshot is one "re im" line per value (src/CrankNicolsonModes_utils.cpp:48-64), each
// number in the default stream format: printf's %g with 6 significant digits, which
// std::to_chars(general, 6) reproduces byte for byte, without the stream machinery.  The
// values are cut into contiguous chunks formatted in parallel and written in order, so the
// file is the one a single std::ofstream would write.
#pragma once

#include <algorithm>
#include <charconv>
#include <complex>
#include <cstddef>
#include <string>
#include <thread>
#include <vector>

// Appends the lines of v[0 .. n) to out.
inline void append_snapshot_lines(std::string &out, const std::complex<double> *v, size_t n)
{
    char buf[64];  // two numbers of at most 13 characters, a space and a newline
    for (size_t k = 0; k < n; ++k) {
        char *p = std::to_chars(buf, buf + 31, v[k].real(), std::chars_format::general, 6).ptr;
        *p++ = ' ';
        p = std::to_chars(p, buf + 62, v[k].imag(), std::chars_format::general, 6).ptr;
        *p++ = '\n';
        out.append(buf, p);
    }
}

// The text of v[0 .. n) in consecutive pieces, formatted by up to `threads` threads.
inline std::vector<std::string> snapshot_text(const std::complex<double> *v, size_t n, unsigned threads)
{
    const size_t parts = std::max<size_t>(1, std::min<size_t>(threads, (n + 65535) / 65536));
    const size_t chunk = (n + parts - 1) / parts;
    std::vector<std::string> text(parts);
    auto run = [&](size_t q) {
        const size_t b = std::min(n, q * chunk), e = std::min(n, b + chunk);
        text[q].reserve((e - b) * 26);
        append_snapshot_lines(text[q], v + b, e - b);
    };
    std::vector<std::thread> pool;
    for (size_t q = 1; q < parts; ++q) pool.emplace_back(run, q);
    run(0);
    for (auto &t : pool) t.join();
    return text;
}
