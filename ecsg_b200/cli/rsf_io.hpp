// rsf_io.hpp -- Madagascar RSF files as the reference's driver reads and writes
// them (iRSF/oRSF of rsf.hh, used by main.cpp, init_del_par_field.cpp,
// init_src.cpp, init_del_rec_trace.cpp, print.cpp and init_del_movie.cpp).
//
// An RSF dataset is a text header of key=value tokens plus float32 samples.
// The samples follow the header in the same file after the bytes 0x0c 0x0c
// 0x04 (in="stdin"), or live in the file named by the header's in= key.
// Only native little-endian float32 (data_format="native_float", esize=4) is
// read or written, which is what the reference's files hold.
#pragma once

#include <cstdio>
#include <map>
#include <string>
#include <utility>
#include <vector>

namespace ecsg_cli {

// key=value tokens of a header text or a command line; later entries win and
// quotes around a value are removed
void parse_pairs(const std::string &text, std::map<std::string, std::string> &kv);

class RsfIn {
public:
    // opens the dataset whose header is at path; throws std::runtime_error
    explicit RsfIn(const std::string &path);
    ~RsfIn();
    RsfIn(const RsfIn &) = delete;
    RsfIn &operator=(const RsfIn &) = delete;

    bool has(const std::string &key) const { return kv_.count(key) != 0; }
    int get_int(const std::string &key, int defolt) const;
    double get_double(const std::string &key, double defolt) const;
    // reads the next n samples; throws if the data ends early
    void read(float *dst, size_t n);
    std::vector<float> read(size_t n);

private:
    std::string path_;
    std::map<std::string, std::string> kv_;
    FILE *data_ = nullptr;
};

class RsfOut {
public:
    // header at path; samples inline after the header (datapath empty) or in
    // datapath/<file name>@ with in= pointing there, as Madagascar's DATAPATH
    RsfOut(const std::string &path, const std::string &datapath);
    ~RsfOut();
    RsfOut(const RsfOut &) = delete;
    RsfOut &operator=(const RsfOut &) = delete;

    // header entries, written in the order given when the first samples are
    // written (oRSF::put); floats use %g like sf_putfloat
    void put(const std::string &key, int v);
    void put(const std::string &key, float v);
    void put(const std::string &key, const std::string &v);
    void write(const float *src, size_t n);
    void close();

private:
    void flush_header();
    std::string path_, datapath_;
    std::vector<std::pair<std::string, std::string>> hdr_;
    FILE *head_ = nullptr, *data_ = nullptr;
    bool started_ = false;
};

} // namespace ecsg_cli
