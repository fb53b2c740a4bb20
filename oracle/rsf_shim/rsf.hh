// rsf.hh -- minimal stand-in for Madagascar's C++ RSF API, written for this
// project so that the reference sources compile unmodified where Madagascar is
// absent.  TEST INFRASTRUCTURE ONLY (oracle build).
//
// Covered surface (exactly what the reference uses):
//   sf_init(argc, argv)                 command line "key=value" parameters
//   iRSF par(0)                         reads parameters from the command line
//   iRSF in("tag")                      opens the RSF file named by tag=<path>
//   iRSF::get(name, value[, default])   int / float / double / bool / string
//   iRSF >> std::valarray<float>        sequential float32 data
//   oRSF out("tag"), type(), put(), << std::valarray<float>
//
// RSF files: a text header of key=value lines.  Data follow either in the same
// file after the bytes 0x0c 0x0c 0x04, or in the file named by the last
// in="..." entry.  Data are little-endian float32 ("native_float").
//
// In-memory inputs: ecsg_rsf_register_memory(tag, header, data, nbytes) makes
// iRSF(tag) read from a caller-owned buffer (used by the oracle driver so that
// large synthetic media need not be written to disk).
#ifndef ECSG_RSF_SHIM_HH
#define ECSG_RSF_SHIM_HH

#include <cstdio>
#include <cstring>
#include <cstdlib>
#include <string>
#include <valarray>
#include <vector>
#include <map>

enum { SF_UCHAR = 0, SF_CHAR, SF_INT, SF_FLOAT, SF_COMPLEX, SF_SHORT, SF_DOUBLE, SF_LONG };

void sf_init(int argc, char *argv[]);

extern "C" void ecsg_rsf_register_memory(const char *tag, const char *header,
                                         const float *data, long nfloats);
extern "C" void ecsg_rsf_clear_memory(void);

class iRSF {
public:
    explicit iRSF(const char *tag = "in");
    explicit iRSF(int);                 // parameter reader (command line)
    ~iRSF();

    void get(const char *name, int &value, int defolt) const;
    void get(const char *name, int &value) const;
    void get(const char *name, float &value, float defolt) const;
    void get(const char *name, float &value) const;
    void get(const char *name, double &value, double defolt) const;
    void get(const char *name, double &value) const;
    void get(const char *name, bool &value, bool defolt) const;
    void get(const char *name, bool &value) const;
    void get(const char *name, std::string &value, const std::string &defolt) const;

    const iRSF &operator>>(std::valarray<float> &array) const;

private:
    bool lookup(const char *name, std::string &out) const;
    std::map<std::string, std::string> kv_;
    bool is_par_;
    mutable FILE *data_;
    const float *mem_;
    mutable long mem_pos_;
    long mem_len_;
};

class oRSF {
public:
    explicit oRSF(const char *tag = "out");
    ~oRSF();
    void type(int t);
    void put(const char *name, int value);
    void put(const char *name, float value);
    void put(const char *name, double value);
    void put(const char *name, const char *value);
    oRSF &operator<<(const std::valarray<float> &array);

private:
    void flush_header();
    std::string path_;
    std::vector<std::pair<std::string, std::string>> kv_;
    FILE *fp_;
    bool header_done_;
    bool sink_;
};

#endif
