// Test harness for the command-line tools' .npy reader and writer
// (cli/cwio.hpp), built and run on the CPU by tests/test_cli_npy.py:
//   cwio_npy read <in.npy> <data.bin>   prints "descr shape..." and writes the raw data
//   cwio_npy write <descr> <data.bin> <out.npy> <dim>...   writes an array of that shape
// Exit status 1 with an ERROR line when the reader refuses a file.
#include <iostream>

#include "cwio.hpp"

int main(int argc, char** argv) {
    try {
        const std::string mode = argc > 1 ? argv[1] : "";
        if (mode == "read" && argc == 4) {
            const cwio::NpyArray a = cwio::read_npy(argv[2]);
            std::cout << a.descr;
            for (size_t s : a.shape) std::cout << ' ' << s;
            std::cout << std::endl;
            std::ofstream f(argv[3], std::ios::binary);
            f.write(a.data.data(), (std::streamsize)a.data.size());
            return 0;
        }
        if (mode == "write" && argc >= 5) {
            std::ifstream f(argv[3], std::ios::binary);
            std::vector<char> data((std::istreambuf_iterator<char>(f)), std::istreambuf_iterator<char>());
            std::vector<size_t> shape;
            for (int i = 5; i < argc; ++i) shape.push_back(std::strtoull(argv[i], nullptr, 10));
            cwio::write_npy(argv[4], argv[2], shape, data.data(), data.size());
            return 0;
        }
        std::cerr << "usage: cwio_npy read in.npy data.bin | write descr data.bin out.npy dims..." << std::endl;
        return 2;
    } catch (const std::exception& e) {
        std::cerr << "ERROR: " << e.what() << std::endl;
        return 1;
    }
}
