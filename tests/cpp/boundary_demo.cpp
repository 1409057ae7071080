// boundary_demo.cpp -- drives libamethyst_b200.so through the C++ mirror (include/amethyst.hpp)
// the way the reference's bench drivers drive its kernels: device buffers owned by the caller,
// the src/lib.cuh launcher names, the survivor count read back after a compressstore
// (src/benchs/bench_compressstore_slabs.cu:38-62).  Test infrastructure: tests/test_cpp_boundary.py
// writes the inputs, runs this program and compares every output with the C oracle.
//
// usage: boundary_demo <dir> <n>
//   inputs  <dir>/a.slab <dir>/b.slab   n elements of 11 bits in slabs
//           <dir>/a.plain64 <dir>/b.plain64 <dir>/a.nogaps <dir>/b.nogaps   the same values
//           <dir>/mask.bin                                                   ceil(n/32) uint32 words
//   outputs <dir>/<name>.out for every operation below
#include <cstdio>
#include <fstream>
#include <string>
#include <vector>

#include "amethyst.hpp"

namespace {

std::vector<uint8_t> slurp(const std::string& p)
{
    std::ifstream f(p, std::ios::binary);
    return std::vector<uint8_t>((std::istreambuf_iterator<char>(f)), std::istreambuf_iterator<char>());
}

void dump(const std::string& p, const void* d_src, size_t bytes)
{
    std::vector<uint8_t> h(bytes);
    if (bytes && cudaMemcpy(h.data(), d_src, bytes, cudaMemcpyDeviceToHost) != cudaSuccess)
        throw amethyst::error(AMX_ERR_CUDA, "copy back failed");
    std::ofstream f(p, std::ios::binary);
    f.write(reinterpret_cast<const char*>(h.data()), (std::streamsize)bytes);
}

void dump_host(const std::string& p, const void* src, size_t bytes)
{
    std::ofstream f(p, std::ios::binary);
    f.write(reinterpret_cast<const char*>(src), (std::streamsize)bytes);
}

template <typename T = uint64_t>
T* upload(const std::vector<uint8_t>& h, size_t capacity)
{
    void* d = nullptr;
    if (cudaMalloc(&d, capacity + 16) != cudaSuccess) throw amethyst::error(AMX_ERR_CUDA, "cudaMalloc failed");
    cudaMemset(d, 0, capacity + 16);
    if (!h.empty()) cudaMemcpy(d, h.data(), h.size(), cudaMemcpyHostToDevice);
    return static_cast<T*>(d);
}

}  // namespace

int main(int argc, char** argv)
{
    if (argc != 3) {
        std::fprintf(stderr, "usage: %s <dir> <n>\n", argv[0]);
        return 2;
    }
    const std::string dir = argv[1];
    const size_t n = std::stoull(argv[2]);
    const size_t big = 8 * n + 64;
    try {
        uint64_t* a_slab = upload(slurp(dir + "/a.slab"), big);
        uint64_t* b_slab = upload(slurp(dir + "/b.slab"), big);
        uint64_t* a_p64 = upload(slurp(dir + "/a.plain64"), big);
        uint64_t* b_p64 = upload(slurp(dir + "/b.plain64"), big);
        uint64_t* a_ng = upload(slurp(dir + "/a.nogaps"), big);
        uint64_t* b_ng = upload(slurp(dir + "/b.nogaps"), big);
        uint8_t* mask = upload<uint8_t>(slurp(dir + "/mask.bin"), big);
        uint64_t* out = upload(std::vector<uint8_t>(), big);
        uint64_t* scal = upload(std::vector<uint8_t>(), 64);

        // the src/lib.cuh launchers
        amethyst::binary_op_slabs<11, 12, AMX_OP_ADD>(a_slab, b_slab, out, n);
        dump(dir + "/add_slab.out", out, amx_storage_bytes(AMX_SLAB, 12, n));
        amethyst::binary_op_nogaps<11, 12, AMX_OP_ADD>(a_ng, b_ng, out, n);
        dump(dir + "/add_nogaps.out", out, amx_storage_bytes(AMX_NOGAPS, 12, n));
        amethyst::binary_op_baseline<11, AMX_OP_MUL>(a_p64, b_p64, out, n);
        dump(dir + "/mul_plain64.out", out, amx_storage_bytes(AMX_PLAIN64, 22, n));
        const size_t cnt = amethyst::compressstore_baseline_cub<11>(mask, a_p64, out, n);
        dump(dir + "/cs_plain64.out", out, amx_storage_bytes(AMX_PLAIN64, 11, cnt));
        uint64_t c64 = cnt;
        dump_host(dir + "/cs_plain64.count", &c64, 8);
        amethyst::filter_baseline<11>(a_p64, out, n, amethyst::pred_half<11>());
        dump(dir + "/filter_half_plain64.out", out, amx_mask_bytes(n));

        // the slab / nogaps forms of the reference's kernels
        amethyst::filter<11>(AMX_SLAB, a_slab, n, out, amethyst::pred(AMX_PRED_LT, 205));
        dump(dir + "/filter_slab.out", out, amx_mask_bytes(n));
        amethyst::compressstore_slabs<11>(mask, a_slab, out, n, scal);
        cudaDeviceSynchronize();
        dump(dir + "/cs_slab.count", scal, 8);
        uint64_t cs = 0;
        cudaMemcpy(&cs, scal, 8, cudaMemcpyDeviceToHost);
        dump(dir + "/cs_slab.out", out, amx_storage_bytes(AMX_SLAB, 11, cs));
        amethyst::hop<11>(AMX_NOGAPS, a_ng, n, scal + 1, AMX_AGG_SUM);
        amethyst::hop<11>(AMX_SLAB, a_slab, n, scal + 2, AMX_AGG_MAX);
        cudaDeviceSynchronize();
        dump(dir + "/hop.out", scal + 1, 16);

        // a program: (a + b) fused into a compressstore of v >= 1024 into 12-bit slabs, then the
        // sum and the minimum of the survivors; run alone, then replayed twice from a graph
        amx_column x{a_slab, n, AMX_SLAB, 11};
        std::vector<amx_step> steps(4);
        steps[0].kind = AMX_STEP_BINARY;
        steps[0].op = AMX_OP_ADD;
        steps[0].value_bits = 12;
        steps[0].out_format = AMX_FORMAT_FUSED;
        steps[0].out_bits = 12;
        steps[0].aux = amx_column{b_slab, n, AMX_SLAB, 11};
        steps[1].kind = AMX_STEP_COMPRESSSTORE;
        steps[1].pred = amethyst::pred(AMX_PRED_GE, 1024);
        steps[1].out_format = AMX_SLAB;
        steps[1].out_bits = 12;
        steps[1].d_result = scal + 3;
        steps[2].kind = AMX_STEP_REDUCE;
        steps[2].op = AMX_AGG_SUM;
        steps[2].d_result = scal + 4;
        steps[3].kind = AMX_STEP_REDUCE;
        steps[3].op = AMX_AGG_MIN;
        steps[3].d_result = scal + 5;
        amethyst::program prog(x, steps);
        prog.run();
        prog.status();
        uint64_t r1[3];
        cudaMemcpy(r1, scal + 3, 24, cudaMemcpyDeviceToHost);
        const uint64_t* d_len = nullptr;
        amx_column fin = prog.output(&d_len);
        uint64_t len = 0;
        cudaMemcpy(&len, d_len, 8, cudaMemcpyDeviceToHost);
        dump(dir + "/program_col.out", fin.data, amx_storage_bytes(fin.format, fin.bits, len));
        dump_host(dir + "/program_res.out", r1, 24);
        cudaMemset(scal + 3, 0, 24);
        amethyst::graph g({&prog}, 1);
        for (int rep = 0; rep < 2; rep++) g.launch();
        cudaDeviceSynchronize();
        uint64_t r2[3];
        cudaMemcpy(r2, scal + 3, 24, cudaMemcpyDeviceToHost);
        dump_host(dir + "/graph_res.out", r2, 24);
        prog.status();

        for (void* p : {(void*)a_slab, (void*)b_slab, (void*)a_p64, (void*)b_p64, (void*)a_ng, (void*)b_ng,
                        (void*)mask, (void*)out, (void*)scal})
            cudaFree(p);
    }
    catch (const amethyst::error& e) {
        std::fprintf(stderr, "amethyst error %d: %s\n", (int)e.status, e.what());
        return 1;
    }
    std::printf("boundary demo ok: n=%zu\n", n);
    return 0;
}
