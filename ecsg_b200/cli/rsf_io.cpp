// rsf_io.cpp -- RSF datasets for the command-line driver (rsf_io.hpp).
#include "rsf_io.hpp"

#include <cstdlib>
#include <cstring>
#include <stdexcept>

namespace ecsg_cli {

namespace {

bool is_space(char c) { return c == ' ' || c == '\t' || c == '\n' || c == '\r'; }

std::string dir_of(const std::string &path)
{
    const size_t s = path.rfind('/');
    return s == std::string::npos ? std::string(".") : path.substr(0, s);
}

std::string base_of(const std::string &path)
{
    const size_t s = path.rfind('/');
    return s == std::string::npos ? path : path.substr(s + 1);
}

} // namespace

void parse_pairs(const std::string &text, std::map<std::string, std::string> &kv)
{
    size_t i = 0;
    const size_t n = text.size();
    while (i < n) {
        while (i < n && is_space(text[i])) i++;
        const size_t s = i;
        bool quoted = false;
        while (i < n && (quoted || !is_space(text[i]))) {
            if (text[i] == '"') quoted = !quoted;
            i++;
        }
        const std::string tok = text.substr(s, i - s);
        const size_t eq = tok.find('=');
        if (eq == std::string::npos || eq == 0) continue;
        std::string v = tok.substr(eq + 1);
        if (v.size() >= 2 && v.front() == '"' && v.back() == '"') v = v.substr(1, v.size() - 2);
        kv[tok.substr(0, eq)] = v;
    }
}

RsfIn::RsfIn(const std::string &path) : path_(path)
{
    FILE *fp = std::fopen(path.c_str(), "rb");
    if (!fp) throw std::runtime_error("cannot open " + path);
    std::string text;
    int c, p1 = -1, p2 = -1;
    bool inline_data = false;
    while ((c = std::fgetc(fp)) != EOF) {
        if (p2 == 0x0c && p1 == 0x0c && c == 0x04) {
            inline_data = true;
            text.resize(text.size() - 2);
            break;
        }
        text.push_back((char)c);
        p2 = p1;
        p1 = c;
    }
    parse_pairs(text, kv_);
    auto fmt = kv_.find("data_format");
    if (fmt != kv_.end() && fmt->second != "native_float") {
        std::fclose(fp);
        throw std::runtime_error(path + ": data_format " + fmt->second + " (only native_float is read)");
    }
    if (get_int("esize", 4) != 4) {
        std::fclose(fp);
        throw std::runtime_error(path + ": esize must be 4");
    }
    if (inline_data) {
        data_ = fp;
        return;
    }
    std::fclose(fp);
    auto in = kv_.find("in");
    if (in == kv_.end() || in->second == "stdin") throw std::runtime_error(path + ": no samples (no in= and no inline data)");
    // in= is relative to the working directory, as in Madagascar; fall back to
    // the header's directory
    data_ = std::fopen(in->second.c_str(), "rb");
    if (!data_ && in->second[0] != '/') data_ = std::fopen((dir_of(path) + "/" + in->second).c_str(), "rb");
    if (!data_) throw std::runtime_error(path + ": cannot open data file " + in->second);
}

RsfIn::~RsfIn()
{
    if (data_) std::fclose(data_);
}

int RsfIn::get_int(const std::string &key, int defolt) const
{
    auto it = kv_.find(key);
    return it == kv_.end() ? defolt : (int)std::strtol(it->second.c_str(), nullptr, 10);
}

double RsfIn::get_double(const std::string &key, double defolt) const
{
    auto it = kv_.find(key);
    return it == kv_.end() ? defolt : std::strtod(it->second.c_str(), nullptr);
}

void RsfIn::read(float *dst, size_t n)
{
    if (std::fread(dst, sizeof(float), n, data_) != n) throw std::runtime_error(path_ + ": fewer samples than the header says");
}

std::vector<float> RsfIn::read(size_t n)
{
    std::vector<float> v(n);
    read(v.data(), n);
    return v;
}

RsfOut::RsfOut(const std::string &path, const std::string &datapath) : path_(path), datapath_(datapath) {}

RsfOut::~RsfOut() { close(); }

void RsfOut::put(const std::string &key, int v) { hdr_.emplace_back(key, std::to_string(v)); }

void RsfOut::put(const std::string &key, float v)
{
    char buf[64];
    std::snprintf(buf, sizeof buf, "%g", (double)v);
    hdr_.emplace_back(key, buf);
}

void RsfOut::put(const std::string &key, const std::string &v) { hdr_.emplace_back(key, "\"" + v + "\""); }

void RsfOut::flush_header()
{
    head_ = std::fopen(path_.c_str(), "wb");
    if (!head_) throw std::runtime_error("cannot create " + path_);
    std::fprintf(head_, "ecsg_main\n");
    for (auto &kv : hdr_) std::fprintf(head_, "\t%s=%s\n", kv.first.c_str(), kv.second.c_str());
    std::fprintf(head_, "\tdata_format=\"native_float\"\n\tesize=4\n");
    if (datapath_.empty()) {
        std::fprintf(head_, "\tin=\"stdin\"\n\n");
        std::fputc(0x0c, head_);
        std::fputc(0x0c, head_);
        std::fputc(0x04, head_);
        data_ = head_;
    } else {
        const std::string bin = datapath_ + "/" + base_of(path_) + "@";
        std::fprintf(head_, "\tin=\"%s\"\n", bin.c_str());
        std::fclose(head_);
        head_ = nullptr;
        data_ = std::fopen(bin.c_str(), "wb");
        if (!data_) throw std::runtime_error("cannot create " + bin);
    }
    started_ = true;
}

void RsfOut::write(const float *src, size_t n)
{
    if (!started_) flush_header();
    if (std::fwrite(src, sizeof(float), n, data_) != n) throw std::runtime_error("write failed: " + path_);
}

void RsfOut::close()
{
    if (!started_ && !path_.empty()) flush_header();   // header-only dataset (no samples)
    if (data_) std::fclose(data_);
    if (head_ && head_ != data_) std::fclose(head_);
    data_ = head_ = nullptr;
    path_.clear();
}

} // namespace ecsg_cli
