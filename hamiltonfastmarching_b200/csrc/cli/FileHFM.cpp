// FileHFM-compatible command-line front-end over the C ABI (include/hfm_b200.h).
//
//   FileHFM_b200 [inputPrefix=input] [outputPrefix=output]
//   FileHFM_<Model> ...   (a link to FileHFM_b200: the solve then requires "model" == <Model>)
//
// Replaces Interfaces/FileHFM/FileHFM.cpp:12-26. Reads <inputPrefix>_Format.txt and the raw float64
// <inputPrefix>_Data.dat in the reference's format (JMM_CPPLibs/JMM_CPPLibs/Output/FileIO.hxx:7-95),
// runs the GPU solve, and writes the computed keys to <outputPrefix>_Format.txt / _Data.dat
// (FileIO.hxx:97-132). On failure prints the message and exits with EXIT_FAILURE.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iostream>
#include <limits>
#include <sstream>
#include <string>
#include <vector>

#include "hfm_b200.h"

namespace {

struct Entry {
    std::string key;
    int depth = 0;  // -1 string, 0 scalar, d array
    std::string str;
    std::vector<int64_t> dims;
    size_t begin = 0, end = 0;
};

bool read_input(const std::string &prefix, hfm_io *io, std::string &err) {
    std::ifstream ifs(prefix + "_Format.txt");
    if (!ifs.is_open()) {
        err = "FileIO error : Input format file could not be opened " + prefix + "_Format.txt.";
        return false;
    }
    auto next_line = [&](std::istream &is) { is.ignore(std::numeric_limits<std::streamsize>::max(), '\n'); };
    std::vector<Entry> entries;
    size_t pos = 0;
    while (!ifs.eof()) {
        Entry e;
        ifs >> e.key;
        next_line(ifs);
        if (e.key.empty()) {
            if (ifs.eof()) break;
            err = "FileIO Error empty field name";
            return false;
        }
        ifs >> e.depth;
        next_line(ifs);
        if (ifs.fail() || e.depth < -1) {
            err = "FileIO error : invalid dimension value for key " + e.key;
            return false;
        }
        if (e.depth == -1) {
            ifs >> e.str;
            next_line(ifs);
        } else {
            size_t size = 1;
            for (int i = 0; i < e.depth; ++i) {
                int64_t d;
                ifs >> d;
                next_line(ifs);
                if (ifs.fail() || d < 0) {
                    err = "FileIO error : invalid dimension for key " + e.key;
                    return false;
                }
                e.dims.push_back(d);
                size *= (size_t)d;
            }
            e.begin = pos;
            e.end = pos + size;
            pos += size;
        }
        next_line(ifs);
        entries.push_back(e);
    }
    std::vector<double> data(pos);
    if (pos) {
        std::ifstream dfs(prefix + "_Data.dat", std::ios::binary);
        if (!dfs.is_open()) {
            err = "FileIO error : input data file could not be opened " + prefix + "_Data.dat";
            return false;
        }
        dfs.seekg(0, dfs.end);
        if ((size_t)dfs.tellg() != pos * sizeof(double)) {
            err = "FileIO error : input data file has incorrect size.";
            return false;
        }
        dfs.seekg(0, dfs.beg);
        dfs.read(reinterpret_cast<char *>(data.data()), pos * sizeof(double));
    }
    for (const Entry &e : entries) {
        int rc;
        if (e.depth == -1) rc = hfm_io_set_string(io, e.key.c_str(), e.str.c_str());
        else if (e.depth == 0) rc = hfm_io_set_scalar(io, e.key.c_str(), data[e.begin]);
        else rc = hfm_io_set_array(io, e.key.c_str(), data.data() + e.begin, e.depth, e.dims.data());
        if (rc != HFM_OK) {
            err = hfm_io_last_error(io);
            return false;
        }
    }
    return true;
}

bool write_output(const std::string &prefix, hfm_io *io, std::string &err) {
    size_t n = 0;
    hfm_io_computed_keys(io, nullptr, 0, &n);
    std::string keys(n + 1, '\0');
    hfm_io_computed_keys(io, &keys[0], n + 1, &n);
    keys.resize(n);
    // "[['key','kind'],...]"
    std::ofstream ofs(prefix + "_Format.txt");
    std::vector<double> out;
    size_t p = 0;
    while ((p = keys.find("['", p)) != std::string::npos) {
        const size_t k0 = p + 2, k1 = keys.find("','", k0);
        const size_t t0 = k1 + 3, t1 = keys.find("']", t0);
        const std::string key = keys.substr(k0, k1 - k0), kind = keys.substr(t0, t1 - t0);
        p = t1;
        ofs << key << "\n";
        if (kind == "string") {
            size_t len = 0;
            hfm_io_get_string(io, key.c_str(), nullptr, 0, &len);
            std::string s(len + 1, '\0');
            hfm_io_get_string(io, key.c_str(), &s[0], len + 1, &len);
            s.resize(len);
            ofs << "-1\n" << s << "\n\n";
        } else if (kind == "float") {
            double v = 0;
            hfm_io_get_scalar(io, key.c_str(), &v);
            ofs << "0\n\n";
            out.push_back(v);
        } else {
            int nd = 0;
            int64_t shape[16];
            hfm_io_get_array_info(io, key.c_str(), &nd, shape, 16);
            size_t size = 1;
            ofs << nd << "\n";
            for (int i = 0; i < nd; ++i) {
                ofs << shape[i] << "\n";
                size *= (size_t)shape[i];
            }
            ofs << "\n";
            const size_t off = out.size();
            out.resize(off + size);
            if (hfm_io_get_array(io, key.c_str(), out.data() + off, size) != HFM_OK) {
                err = hfm_io_last_error(io);
                return false;
            }
        }
    }
    std::ofstream dfs(prefix + "_Data.dat", std::ios::binary);
    dfs.write(reinterpret_cast<const char *>(out.data()), out.size() * sizeof(double));
    return true;
}

}  // namespace

int main(int argc, const char *argv[]) {
    const std::string in = argc > 1 ? argv[1] : "input", out = argc > 2 ? argv[2] : "output";
    std::string exe = argv[0];
    const size_t slash = exe.find_last_of('/');
    if (slash != std::string::npos) exe = exe.substr(slash + 1);
    std::string expected;
    if (exe.rfind("FileHFM_", 0) == 0 && exe != "FileHFM_b200") expected = exe.substr(8);
    hfm_io *io = hfm_io_create(HFM_ORDER_ROW_MAJOR);
    if (!io) return EXIT_FAILURE;
    std::string err;
    int code = EXIT_SUCCESS;
    if (!read_input(in, io, err)) {
        code = EXIT_FAILURE;
    } else if (hfm_run(io, expected.empty() ? nullptr : expected.c_str()) != HFM_OK) {
        err = hfm_io_last_error(io);
        code = EXIT_FAILURE;
    }
    if (code != EXIT_SUCCESS)
        std::cout << "***** Warning ! *****\nException caught. " << err << "\n********************\n";
    std::string werr;
    if (!write_output(out, io, werr)) {
        std::cout << werr << "\n";
        code = EXIT_FAILURE;
    }
    hfm_io_destroy(io);
    return code;
}
