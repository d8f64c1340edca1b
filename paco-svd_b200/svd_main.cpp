// svd_main: command-line driver with the file contract of the reference's
// main.cpp (DEAVEN-MITCH/paco-svd main.cpp:15-203):
//   reads "M N" from ../args.txt (main.cpp:20-24) and the raw little-endian
//   FP32 row-major M x N matrix ../input/A_gm.bin (main.cpp:64), runs both
//   stages on the GPU, writes ../output/sigma.bin (N floats, descending),
//   ../output/U.bin (M x M) and ../output/Vt.bin (N x N) (main.cpp:171-174).
// Options --args FILE, --input FILE, --output DIR override those paths.
// Unlike the reference (which logs and continues, data_utils.h:41-47), any
// failure exits with a non-zero status.
#include <sys/stat.h>

#include <cstdio>
#include <cstring>
#include <fstream>
#include <iostream>
#include <string>
#include <vector>

#include "paco_svd.h"

static bool read_file(const std::string &path, void *buf, size_t bytes)
{
    std::ifstream f(path, std::ios::binary);
    if (!f) {
        std::cerr << "[ERROR] cannot open " << path << "\n";
        return false;
    }
    f.seekg(0, std::ios::end);
    size_t size = (size_t)f.tellg();
    f.seekg(0);
    if (size < bytes) {
        std::cerr << "[ERROR] " << path << " holds " << size << " bytes, expected " << bytes << "\n";
        return false;
    }
    if (size > bytes) std::cerr << "[WARN] " << path << " is larger than the buffer, reading " << bytes << " bytes\n";
    f.read((char *)buf, (std::streamsize)bytes);
    return (bool)f;
}

static bool write_file(const std::string &path, const void *buf, size_t bytes)
{
    std::ofstream f(path, std::ios::binary | std::ios::trunc);
    if (!f) {
        std::cerr << "[ERROR] cannot write " << path << "\n";
        return false;
    }
    f.write((const char *)buf, (std::streamsize)bytes);
    return (bool)f;
}

int main(int argc, char **argv)
{
    std::string args_path = "../args.txt", in_path = "../input/A_gm.bin", out_dir = "../output";
    for (int i = 1; i + 1 < argc; i += 2) {
        if (!strcmp(argv[i], "--args")) args_path = argv[i + 1];
        else if (!strcmp(argv[i], "--input")) in_path = argv[i + 1];
        else if (!strcmp(argv[i], "--output")) out_dir = argv[i + 1];
        else {
            std::cerr << "usage: svd_main [--args FILE] [--input FILE] [--output DIR]\n";
            return 2;
        }
    }
    std::ifstream af(args_path);
    long M = 0, N = 0;
    if (!(af >> M >> N)) {
        std::cerr << "[ERROR] cannot read \"M N\" from " << args_path << "\n";
        return 1;
    }
    if (M < N) {
        std::cerr << "M must be greater than N" << std::endl;
        return 1;
    }
    std::vector<float> A((size_t)M * N), U((size_t)M * M), Vt((size_t)N * N), sigma((size_t)N);
    if (!read_file(in_path, A.data(), A.size() * sizeof(float))) return 1;
    paco_ctx *ctx = nullptr;
    int rc = paco_ctx_create((int)M, (int)N, &ctx);
    if (rc) {
        std::cerr << "[ERROR] paco_ctx_create failed with status " << rc << "\n";
        return 1;
    }
    std::cout << "before svd" << std::endl;
    rc = paco_ctx_svd_host(ctx, A.data(), U.data(), Vt.data(), sigma.data());
    paco_ctx_destroy(ctx);
    if (rc) {
        std::cerr << "[ERROR] SVD failed with status " << rc << "\n";
        return 1;
    }
    std::cout << "finish" << std::endl;
    mkdir(out_dir.c_str(), 0755);
    bool ok = write_file(out_dir + "/sigma.bin", sigma.data(), sigma.size() * sizeof(float)) &&
              write_file(out_dir + "/U.bin", U.data(), U.size() * sizeof(float)) &&
              write_file(out_dir + "/Vt.bin", Vt.data(), Vt.size() * sizeof(float));
    return ok ? 0 : 1;
}
