// A C++ caller of the reference-shaped facade (include/cbs_b200.hpp) linked against
// libcbs_b200.so: the program a Phantom / CirBTS user would write, run by
// tests/test_cpp_facade_gpu.py, which supplies the inputs and checks the outputs against the
// oracle.  Modes (argv[1]), files in the directory argv[2]:
//   ks    keyswitch_inplace through EncryptionParameters / PhantomContext / PhantomCiphertext /
//         PhantomRelinKey: ks_dims (N size_q size_p chain_index beta), ks_chain, ks_c2, ks_ct,
//         ks_evk -> ks_out
//   cbs   GPUCirBTSContext: KeyGen(seed), gpu_CircuitBootstrappingBatch, gpu_CircuitBootstrapping and
//         gpu_CircuitBootstrappingBatchToDevice on host LWE ciphertexts: cbs_dims (seed batch
//         [backend]), cbs_a, cbs_b -> cbs_out (the batch's RGSW rows)
//   gate  GPUBinFHEContext::BatchGPUEvalBinGate(NAND): exit status 0 when every gate decrypts to
//         the truth table
//   gfunc GPUBinFHEContext's functional evaluators (BatchGPUEvalFunc, GPUEvalFunc, BatchGPUEvalSign,
//         BatchGPUEvalFloor, BatchGPUEvalDecomp): exit status 0 when every result decrypts right
//   lmk   GPUCirBTSContext with SetMethod(LMKCDEY): gpu_CircuitBootstrappingBatch on the 2^18 x 2
//         preset with one LUT slot, and LMKCDEY_EvalAcc on a given accumulator: lmk_dims (seed
//         batch num_auto_keys), lmk_a, lmk_b, lmk_acc, lmk_masks -> lmk_cbs_out, lmk_acc_out
//   ckks  the CKKS evaluator: multiply_and_relin_inplace then rescale_to_next_inplace of ct1 by
//         ct2, and rotate_inplace of ct1 by one step: ck_dims (N size_q size_p chain_index beta
//         galois_elt), ck_chain, ck_ct1, ck_ct2, ck_rk, ck_gk -> ck_mr, ck_rot
#include <algorithm>
#include <cstdio>
#include <fstream>
#include <iostream>
#include <string>
#include <vector>

#include "cbs_b200.hpp"

using namespace cbs_b200;

template <class T>
static std::vector<T> read_raw(const std::string& path) {
    std::ifstream f(path, std::ios::binary | std::ios::ate);
    if (!f) throw std::runtime_error("cannot open " + path);
    const std::streamsize bytes = f.tellg();
    f.seekg(0);
    std::vector<T> v(static_cast<size_t>(bytes) / sizeof(T));
    f.read(reinterpret_cast<char*>(v.data()), bytes);
    return v;
}

template <class T>
static void write_raw(const std::string& path, const std::vector<T>& v) {
    std::ofstream f(path, std::ios::binary);
    f.write(reinterpret_cast<const char*>(v.data()), static_cast<std::streamsize>(v.size() * sizeof(T)));
}

static int run_ks(const std::string& dir) {
    const auto dims = read_raw<uint64_t>(dir + "/ks_dims");
    const size_t N = dims[0], size_q = dims[1], size_p = dims[2], chain_index = dims[3], beta = dims[4];
    const auto chain = read_raw<uint64_t>(dir + "/ks_chain");
    phantom::EncryptionParameters parms(phantom::scheme_type::ckks);
    parms.set_poly_modulus_degree(N);
    parms.set_coeff_modulus(chain);
    parms.set_special_modulus_size(size_p);
    PhantomContext context(parms);
    cudaStream_t stream = nullptr;
    check_cuda(cudaStreamCreate(&stream), "stream");
    PhantomCiphertext ct;
    ct.resize(context, chain_index, 2, stream);
    const size_t size_ql = ct.coeff_modulus_size();
    if (size_ql != size_q - (chain_index - 1)) return 3;
    const auto h_ct = read_raw<uint64_t>(dir + "/ks_ct");
    const auto h_c2 = read_raw<uint64_t>(dir + "/ks_c2");
    if (h_ct.size() != 2 * size_ql * N || h_c2.size() != size_ql * N) return 4;
    check_cuda(cudaMemcpy(ct.data(), h_ct.data(), h_ct.size() * 8, cudaMemcpyHostToDevice), "ct in");
    DeviceArray<uint64_t> c2(h_c2.size());
    check_cuda(cudaMemcpy(c2.data(), h_c2.data(), h_c2.size() * 8, cudaMemcpyHostToDevice), "c2 in");
    PhantomRelinKey relin(context, read_raw<uint64_t>(dir + "/ks_evk"), beta);
    keyswitch_inplace(context, ct, c2.data(), relin, false, stream);
    std::vector<uint64_t> out(h_ct.size());
    check_cuda(cudaStreamSynchronize(stream), "sync");
    check_cuda(cudaMemcpy(out.data(), ct.data(), out.size() * 8, cudaMemcpyDeviceToHost), "ct out");
    write_raw(dir + "/ks_out", out);
    cudaStreamDestroy(stream);
    return 0;
}

static int run_cbs(const std::string& dir) {
    const auto dims = read_raw<uint64_t>(dir + "/cbs_dims");
    const uint64_t seed = dims[0];
    const uint32_t batch = static_cast<uint32_t>(dims[1]);
    cbs_params params{};
    check(cbs_params_default(&params), "params");
    GPUCirBTSContext cc(params, batch);
    if (dims.size() > 2) cc.SetBackend(static_cast<int>(dims[2]));  // default: the context's (NTT)
    cc.KeyGen(seed);
    const auto a = read_raw<uint64_t>(dir + "/cbs_a");
    const auto b = read_raw<uint64_t>(dir + "/cbs_b");
    std::vector<LWECiphertext> cts(batch);
    for (uint32_t i = 0; i < batch; ++i) {
        cts[i].a.assign(a.begin() + static_cast<size_t>(i) * params.n, a.begin() + static_cast<size_t>(i + 1) * params.n);
        cts[i].b = b[i];
        cts[i].q = params.q_lwe;
    }
    const auto rgsw = cc.gpu_CircuitBootstrappingBatch(cts);
    std::vector<uint64_t> out;
    for (const auto& r : rgsw) out.insert(out.end(), r.data.begin(), r.data.end());
    write_raw(dir + "/cbs_out", out);
    // the single-ciphertext and device-view forms agree with the batch
    const auto one = cc.gpu_CircuitBootstrapping(cts[batch - 1]);
    if (one.data != rgsw[batch - 1].data) return 5;
    const auto view = cc.gpu_CircuitBootstrappingBatchToDevice(cts);
    std::vector<uint64_t> back(view.per_ciphertext_elems * view.batch);
    check_cuda(cudaStreamSynchronize(view.stream), "sync");
    check_cuda(cudaMemcpy(back.data(), view.d_rgsw, back.size() * 8, cudaMemcpyDeviceToHost), "view");
    if (back != out) return 6;
    // a ciphertext of another modulus is rejected with an exception
    try {
        LWECiphertext bad = cts[0];
        bad.q = params.q_lwe * 2;
        (void)cc.gpu_CircuitBootstrapping(bad);
        return 7;
    } catch (const Error&) {
    }
    return 0;
}

static int run_lmk(const std::string& dir) {
    const auto dims = read_raw<uint64_t>(dir + "/lmk_dims");
    const uint64_t seed = dims[0];
    const uint32_t batch = static_cast<uint32_t>(dims[1]), num_auto = static_cast<uint32_t>(dims[2]);
    cbs_params params{};
    check(cbs_params_preset(CBS_PARAMS_AES_2X18, &params), "params");
    params.num_lut = 1;
    GPUCirBTSContext cc(params, batch);
    cc.SetMethod(CBS_BR_LMKCDEY, num_auto);
    cc.KeyGen(seed);
    const auto a = read_raw<uint64_t>(dir + "/lmk_a");
    const auto b = read_raw<uint64_t>(dir + "/lmk_b");
    std::vector<LWECiphertext> cts(batch);
    for (uint32_t i = 0; i < batch; ++i) {
        cts[i].a.assign(a.begin() + static_cast<size_t>(i) * params.n, a.begin() + static_cast<size_t>(i + 1) * params.n);
        cts[i].b = b[i];
        cts[i].q = params.q_lwe;
    }
    const auto rgsw = cc.gpu_CircuitBootstrappingBatch(cts);
    std::vector<uint64_t> out;
    for (const auto& r : rgsw) out.insert(out.end(), r.data.begin(), r.data.end());
    write_raw(dir + "/lmk_cbs_out", out);
    // EvalAcc on a given accumulator and masks
    const auto acc = read_raw<uint64_t>(dir + "/lmk_acc");
    const auto masks = read_raw<uint32_t>(dir + "/lmk_masks");
    DeviceArray<uint64_t> d_acc(acc.size());
    check_cuda(cudaMemcpy(d_acc.data(), acc.data(), acc.size() * 8, cudaMemcpyHostToDevice), "acc in");
    cc.LMKCDEY_EvalAcc(masks, d_acc.data());
    std::vector<uint64_t> acc_out(acc.size());
    check_cuda(cudaMemcpy(acc_out.data(), d_acc.data(), acc.size() * 8, cudaMemcpyDeviceToHost), "acc out");
    write_raw(dir + "/lmk_acc_out", acc_out);
    return 0;
}

static int run_gate(const std::string&) {
    cbs_gate_params gp{};
    check(cbs_gate_params_default(&gp), "gate params");
    GPUBinFHEContext cc(gp, 64);
    cc.GPUBTKeyGen(17);
    const uint32_t count = 16;
    std::vector<uint8_t> x(count), y(count);
    for (uint32_t i = 0; i < count; ++i) x[i] = i & 1, y[i] = (i >> 1) & 1;
    std::vector<uint32_t> a1(count * gp.n), b1(count), a2(count * gp.n), b2(count);
    check(cbs_gate_encrypt_bits(cc.handle(), x.data(), count, 1, a1.data(), b1.data()), "encrypt");
    check(cbs_gate_encrypt_bits(cc.handle(), y.data(), count, 2, a2.data(), b2.data()), "encrypt");
    auto wrap = [&](const std::vector<uint32_t>& a, const std::vector<uint32_t>& b) {
        std::vector<LWECiphertext> v(count);
        for (uint32_t i = 0; i < count; ++i) {
            v[i].a.assign(a.begin() + static_cast<size_t>(i) * gp.n, a.begin() + static_cast<size_t>(i + 1) * gp.n);
            v[i].b = b[i];
            v[i].q = uint64_t(1) << 32;
        }
        return v;
    };
    const auto out = cc.BatchGPUEvalBinGate(NAND, wrap(a1, b1), wrap(a2, b2));
    std::vector<uint32_t> oa(count * gp.n), ob(count);
    for (uint32_t i = 0; i < count; ++i) {
        for (uint32_t j = 0; j < gp.n; ++j) oa[static_cast<size_t>(i) * gp.n + j] = static_cast<uint32_t>(out[i].a[j]);
        ob[i] = static_cast<uint32_t>(out[i].b);
    }
    std::vector<uint8_t> dec(count);
    check(cbs_gate_decrypt_bits(cc.handle(), oa.data(), ob.data(), count, dec.data()), "decrypt");
    for (uint32_t i = 0; i < count; ++i)
        if (dec[i] != static_cast<uint8_t>(1 - (x[i] & y[i]))) return 8;
    return 0;
}

// LWE encryption of phases mod q under s (test helper: the facade's user holds s)
static std::vector<LWECiphertext> encrypt_mod(const std::vector<int32_t>& s, const std::vector<uint64_t>& phases,
                                              uint64_t q, uint64_t seed) {
    uint64_t x = seed;
    auto next = [&]() {  // splitmix64
        uint64_t z = (x += 0x9e3779b97f4a7c15ull);
        z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
        z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
        return z ^ (z >> 31);
    };
    std::vector<LWECiphertext> v(phases.size());
    for (size_t i = 0; i < phases.size(); ++i) {
        v[i].a.resize(s.size());
        uint64_t dot = 0;
        for (size_t j = 0; j < s.size(); ++j) {
            v[i].a[j] = next() & (q - 1);
            dot += v[i].a[j] * static_cast<uint64_t>(s[j]);
        }
        v[i].b = (dot + phases[i] + (next() % 3) - 1) & (q - 1);  // noise in {-1, 0, 1}
        v[i].q = q;
    }
    return v;
}

static uint64_t phase_of(const std::vector<int32_t>& s, const LWECiphertext& c) {
    uint64_t dot = 0;
    for (size_t j = 0; j < s.size(); ++j) dot += c.a[j] * static_cast<uint64_t>(s[j]);
    return (c.b - dot) & (c.q - 1);
}

static int run_gfunc(const std::string&) {
    cbs_gate_params gp{};
    check(cbs_gate_params_default(&gp), "gate params");
    GPUBinFHEContext cc(gp, 16);
    cc.GPUBTKeyGen(23);
    cc.SetFunctionalParams(1024, 128);
    std::vector<int32_t> s(gp.n);
    check(cbs_gate_export_keys(cc.handle(), s.data(), nullptr, nullptr, nullptr), "keys");
    // EvalFunc of x -> 3x mod 4 (an arbitrary table) on q = 1024
    const uint64_t q = 1024, P = 4;
    std::vector<uint64_t> lut(q);
    for (uint64_t x = 0; x < q; ++x) lut[x] = (q / P) * ((3 * ((x * P) / q)) % P);
    std::vector<uint64_t> ms = {0, 1, 2, 3}, ph;
    for (auto m : ms) ph.push_back(m * (q / P));
    const auto fo = cc.BatchGPUEvalFunc(encrypt_mod(s, ph, q, 1), lut);
    for (size_t i = 0; i < ms.size(); ++i)
        if (((phase_of(s, fo[i]) + q / (2 * P)) / (q / P)) % P != (3 * ms[i]) % P) return 20;
    if (cc.GPUEvalFunc(encrypt_mod(s, {ph[1]}, q, 2)[0], lut).q != q) return 21;
    // EvalSign of 14-bit values: output mod q, 0 below 2^13 and q/2 above
    const uint64_t mod = uint64_t(1) << 14;
    const std::vector<uint64_t> xs = {1000, 7000, 9000, 15000};
    const auto sg = cc.BatchGPUEvalSign(encrypt_mod(s, xs, mod, 3));
    for (size_t i = 0; i < xs.size(); ++i) {
        const uint64_t p = phase_of(s, sg[i]), want = xs[i] >= mod / 2 ? q / 2 : 0;
        const uint64_t d = (p - want) & (q - 1);
        if (std::min(d, q - d) >= q / 8) return 22;
    }
    // EvalFloor keeps the modulus; EvalDecomp gives three digits for 14 bits at q = 2^10, beta = 2^7
    if (cc.BatchGPUEvalFloor(encrypt_mod(s, xs, mod, 4))[0].q != mod) return 23;
    const auto dg = cc.BatchGPUEvalDecomp(encrypt_mod(s, xs, mod, 5));
    if (dg.size() != xs.size() || dg[0].size() != 3) return 24;
    for (size_t i = 0; i < xs.size(); ++i) {
        const uint64_t d = (phase_of(s, dg[i][0]) - xs[i]) & (q - 1);
        if (std::min(d, q - d) >= 32) return 25;
    }
    return 0;
}

static int run_ckks(const std::string& dir) {
    const auto dims = read_raw<uint64_t>(dir + "/ck_dims");
    const size_t N = dims[0], size_p = dims[2], chain_index = dims[3], beta = dims[4];
    const uint32_t elt = static_cast<uint32_t>(dims[5]);
    phantom::EncryptionParameters parms(phantom::scheme_type::ckks);
    parms.set_poly_modulus_degree(N);
    parms.set_coeff_modulus(read_raw<uint64_t>(dir + "/ck_chain"));
    parms.set_special_modulus_size(size_p);
    PhantomContext context(parms);
    const cudaStream_t stream = nullptr;
    auto load_ct = [&](const std::string& name, PhantomCiphertext& ct) {
        ct.resize(context, chain_index, 2, stream);
        const auto h = read_raw<uint64_t>(dir + "/" + name);
        if (h.size() != 2 * ct.coeff_modulus_size() * N) throw std::runtime_error("ciphertext size");
        check_cuda(cudaMemcpy(ct.data(), h.data(), h.size() * 8, cudaMemcpyHostToDevice), "ct in");
    };
    auto save_ct = [&](const std::string& name, const PhantomCiphertext& ct) {
        std::vector<uint64_t> h(ct.size() * ct.coeff_modulus_size() * N);
        check_cuda(cudaDeviceSynchronize(), "sync");
        check_cuda(cudaMemcpy(h.data(), ct.data(), h.size() * 8, cudaMemcpyDeviceToHost), "ct out");
        write_raw(dir + "/" + name, h);
    };
    PhantomCiphertext ct1, ct2, ct3;
    load_ct("ck_ct1", ct1);
    load_ct("ck_ct2", ct2);
    load_ct("ck_ct1", ct3);
    PhantomRelinKey relin(context, read_raw<uint64_t>(dir + "/ck_rk"), beta);
    PhantomGaloisKey galois;
    galois.insert(elt, PhantomRelinKey(context, read_raw<uint64_t>(dir + "/ck_gk"), beta));
    multiply_and_relin_inplace(context, ct1, ct2, relin);
    const size_t limbs = ct1.coeff_modulus_size();
    rescale_to_next_inplace(context, ct1, static_cast<double>(read_raw<uint64_t>(dir + "/ck_chain")[limbs - 1]));
    if (ct1.chain_index() != chain_index + 1 || ct1.size() != 2) return 5;
    save_ct("ck_mr", ct1);
    rotate_inplace(context, ct3, 1, galois);
    save_ct("ck_rot", ct3);
    return 0;
}

int main(int argc, char** argv) {
    if (argc < 3) {
        std::fprintf(stderr, "usage: %s ks|cbs|gate|ckks|lmk|gfunc <dir>\n", argv[0]);
        return 2;
    }
    try {
        const std::string mode = argv[1], dir = argv[2];
        if (mode == "ks") return run_ks(dir);
        if (mode == "cbs") return run_cbs(dir);
        if (mode == "gate") return run_gate(dir);
        if (mode == "ckks") return run_ckks(dir);
        if (mode == "lmk") return run_lmk(dir);
        if (mode == "gfunc") return run_gfunc(dir);
    } catch (const std::exception& e) {
        std::fprintf(stderr, "error: %s\n", e.what());
        return 1;
    }
    return 2;
}
