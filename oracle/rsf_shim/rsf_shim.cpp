// rsf_shim.cpp -- implementation of the project-written RSF stand-in (rsf.hh).
// TEST INFRASTRUCTURE ONLY (oracle build).
#include "rsf.hh"

#include <cerrno>
#include <iostream>

namespace {
std::map<std::string, std::string> &cli()
{
    static std::map<std::string, std::string> m;
    return m;
}
struct MemFile {
    std::string header;
    const float *data;
    long n;
};
std::map<std::string, MemFile> &mem()
{
    static std::map<std::string, MemFile> m;
    return m;
}

void fail(const std::string &msg)
{
    std::cerr << "rsf shim: " << msg << std::endl;
    std::exit(2);
}

std::string unquote(std::string v)
{
    if (v.size() >= 2 && v.front() == '"' && v.back() == '"') v = v.substr(1, v.size() - 2);
    return v;
}

// Parse "key=value" tokens of a header text; later entries win.
void parse_header(const std::string &text, std::map<std::string, std::string> &kv)
{
    size_t i = 0, n = text.size();
    while (i < n) {
        while (i < n && (text[i] == ' ' || text[i] == '\t' || text[i] == '\n' || text[i] == '\r')) i++;
        size_t s = i;
        bool inq = false;
        while (i < n && (inq || (text[i] != ' ' && text[i] != '\t' && text[i] != '\n' && text[i] != '\r'))) {
            if (text[i] == '"') inq = !inq;
            i++;
        }
        std::string tok = text.substr(s, i - s);
        size_t eq = tok.find('=');
        if (eq != std::string::npos && eq > 0) kv[tok.substr(0, eq)] = unquote(tok.substr(eq + 1));
    }
}
} // namespace

void sf_init(int argc, char *argv[])
{
    cli().clear();
    for (int i = 1; i < argc; i++) {
        std::string a(argv[i]);
        size_t eq = a.find('=');
        if (eq != std::string::npos) cli()[a.substr(0, eq)] = unquote(a.substr(eq + 1));
    }
}

extern "C" void ecsg_rsf_register_memory(const char *tag, const char *header, const float *data, long n)
{
    mem()[tag] = MemFile{header ? header : "", data, n};
}
extern "C" void ecsg_rsf_clear_memory(void) { mem().clear(); }

iRSF::iRSF(int) : is_par_(true), data_(nullptr), mem_(nullptr), mem_pos_(0), mem_len_(0)
{
    kv_ = cli();
}

iRSF::iRSF(const char *tag) : is_par_(false), data_(nullptr), mem_(nullptr), mem_pos_(0), mem_len_(0)
{
    auto m = mem().find(tag);
    if (m != mem().end()) {
        parse_header(m->second.header, kv_);
        mem_ = m->second.data;
        mem_len_ = m->second.n;
        return;
    }
    auto it = cli().find(tag);
    if (it == cli().end()) fail(std::string("no file given for tag '") + tag + "'");
    FILE *fp = std::fopen(it->second.c_str(), "rb");
    if (!fp) fail("cannot open " + it->second);
    std::string text;
    int c, prev2 = -1, prev1 = -1;
    bool inline_data = false;
    while ((c = std::fgetc(fp)) != EOF) {
        if (prev2 == 0x0c && prev1 == 0x0c && c == 0x04) { inline_data = true; break; }
        prev2 = prev1; prev1 = c;
        text.push_back((char)c);
    }
    parse_header(text, kv_);
    if (inline_data) {
        data_ = fp;
    } else {
        std::fclose(fp);
        auto in = kv_.find("in");
        if (in == kv_.end()) fail("no data for " + it->second);
        data_ = std::fopen(in->second.c_str(), "rb");
        if (!data_) fail("cannot open data file " + in->second);
    }
}

iRSF::~iRSF()
{
    if (data_) std::fclose(data_);
}

bool iRSF::lookup(const char *name, std::string &out) const
{
    auto it = kv_.find(name);
    if (it == kv_.end()) return false;
    out = it->second;
    return true;
}

void iRSF::get(const char *name, int &value, int defolt) const
{
    std::string s;
    value = lookup(name, s) ? (int)std::strtol(s.c_str(), nullptr, 10) : defolt;
}
void iRSF::get(const char *name, int &value) const
{
    std::string s;
    if (lookup(name, s)) value = (int)std::strtol(s.c_str(), nullptr, 10);
}
void iRSF::get(const char *name, float &value, float defolt) const
{
    std::string s;
    value = lookup(name, s) ? std::strtof(s.c_str(), nullptr) : defolt;
}
void iRSF::get(const char *name, float &value) const
{
    std::string s;
    if (lookup(name, s)) value = std::strtof(s.c_str(), nullptr);
}
void iRSF::get(const char *name, double &value, double defolt) const
{
    std::string s;
    value = lookup(name, s) ? std::strtod(s.c_str(), nullptr) : defolt;
}
void iRSF::get(const char *name, double &value) const
{
    std::string s;
    if (lookup(name, s)) value = std::strtod(s.c_str(), nullptr);
}
void iRSF::get(const char *name, bool &value, bool defolt) const
{
    std::string s;
    if (!lookup(name, s)) { value = defolt; return; }
    value = !s.empty() && (s[0] == 'y' || s[0] == 'Y' || s[0] == '1' || s[0] == 't' || s[0] == 'T');
}
void iRSF::get(const char *name, bool &value) const
{
    get(name, value, value);
}
void iRSF::get(const char *name, std::string &value, const std::string &defolt) const
{
    std::string s;
    value = lookup(name, s) ? s : defolt;
}

const iRSF &iRSF::operator>>(std::valarray<float> &array) const
{
    size_t n = array.size();
    if (mem_) {
        if (mem_pos_ + (long)n > mem_len_) fail("read past end of in-memory input");
        for (size_t i = 0; i < n; i++) array[i] = mem_[mem_pos_ + i];
        mem_pos_ += (long)n;
        return *this;
    }
    if (!data_) fail("read from a parameter reader");
    if (n && std::fread(&array[0], sizeof(float), n, data_) != n) fail("short read");
    return *this;
}

oRSF::oRSF(const char *tag) : fp_(nullptr), header_done_(false), sink_(false)
{
    auto it = cli().find(tag);
    if (it == cli().end()) { sink_ = true; return; }
    path_ = it->second;
    fp_ = std::fopen(path_.c_str(), "wb");
    if (!fp_) fail("cannot create " + path_);
}

oRSF::~oRSF()
{
    if (fp_) {
        flush_header();
        std::fclose(fp_);
    }
}

void oRSF::type(int) { kv_.push_back({"data_format", "\"native_float\""}); kv_.push_back({"esize", "4"}); }
void oRSF::put(const char *name, int value) { kv_.push_back({name, std::to_string(value)}); }
void oRSF::put(const char *name, float value)
{
    char b[64];
    std::snprintf(b, sizeof b, "%.9g", (double)value);
    kv_.push_back({name, b});
}
void oRSF::put(const char *name, double value)
{
    char b[64];
    std::snprintf(b, sizeof b, "%.17g", value);
    kv_.push_back({name, b});
}
void oRSF::put(const char *name, const char *value) { kv_.push_back({name, std::string("\"") + value + "\""}); }

void oRSF::flush_header()
{
    if (header_done_ || !fp_) return;
    for (auto &p : kv_) std::fprintf(fp_, "\t%s=%s\n", p.first.c_str(), p.second.c_str());
    std::fputc(0x0c, fp_);
    std::fputc(0x0c, fp_);
    std::fputc(0x04, fp_);
    header_done_ = true;
}

oRSF &oRSF::operator<<(const std::valarray<float> &array)
{
    if (sink_) return *this;
    flush_header();
    if (array.size()) std::fwrite(&array[0], sizeof(float), array.size(), fp_);
    return *this;
}
