// Drives the cusignal:: C++ API (include/cusignal/...) the way the reference's callers
// do -- pulse compression, resident pulse Doppler, cfar_alpha, CA-CFAR, firfilter,
// upfirdn, resample_poly, firfilter2, hilbert, the batched FFT -- on inputs read from <dir>/*.bin and writes
// every result to <dir>/out_*.bin for tests/test_gpu_dropin.py to check.
#include <cusignal/operators/filtering/filtering_typed.h>
#include <cusignal/operators/radartools/radartools_typed.h>
#include <cusignal/runtime/cuda_utils.h>

#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <iostream>
#include <string>
#include <vector>

namespace {
std::string g_dir;

template <class T>
std::vector<T> load(const std::string& name)
{
    std::ifstream f(g_dir + "/" + name, std::ios::binary | std::ios::ate);
    if (!f) throw std::runtime_error("missing input " + name);
    const std::streamsize bytes = f.tellg();
    f.seekg(0);
    std::vector<T> v(static_cast<std::size_t>(bytes) / sizeof(T));
    f.read(reinterpret_cast<char*>(v.data()), bytes);
    return v;
}

template <class T>
void save(const std::string& name, const std::vector<T>& v)
{
    std::ofstream f(g_dir + "/out_" + name + ".bin", std::ios::binary);
    f.write(reinterpret_cast<const char*>(v.data()), static_cast<std::streamsize>(v.size() * sizeof(T)));
}
}  // namespace

int main(int argc, char** argv)
{
    if (argc != 2) {
        std::cerr << "usage: dropin_probe <dir>\n";
        return 2;
    }
    g_dir = argv[1];
    try {
        using namespace cusignal;
        const auto dims = load<int>("dims.bin");  // P, N, L, nfir, ntaps
        const int P = dims[0], N = dims[1], L = dims[2], NF = dims[3], NT = dims[4];
        auto x = DeviceArray<TypedComplex<float>>::from_host(load<TypedComplex<float>>("x.bin"));
        auto t = DeviceArray<TypedComplex<float>>::from_host(load<TypedComplex<float>>("t.bin"));

        // step 2 of the chain: windowed, normalised compression (FP64 storage result)
        PulseCompressionOptions pc;
        pc.num_pulses = P;
        pc.samples_per_pulse = N;
        pc.normalize = true;
        pc.window = RadarWindowKind::hamming;
        auto comp = pulse_compression_device(x, t, pc);
        if (!comp.is_fp64) throw std::runtime_error("windowed compression must return FP64 storage");
        save("pc", comp.fp64.to_host());

        // step 3: resident Doppler of the FP32 compression of the same data
        pc.window = RadarWindowKind::none;
        auto comp32 = pulse_compression_device(x, t, pc);
        if (comp32.is_fp64) throw std::runtime_error("unwindowed FP32 compression must stay FP32");
        save("pc32", comp32.fp32.to_host());
        PulseDopplerOptions pd;
        pd.num_pulses = P;
        pd.samples_per_pulse = N;
        pd.window = RadarWindowKind::hamming;
        DeviceArray<ComplexFloat> rd(static_cast<std::size_t>(P) * N);
        DeviceArray<TypedComplex<float>> comp_view(comp32.fp32.size());
        cuda_utils::copy_device_to_device(reinterpret_cast<ComplexFloat*>(comp_view.data()), comp32.fp32.data(),
                                          comp32.fp32.size());
        pulse_doppler_device(comp_view, pd, rd);
        auto rdh = rd.to_host();
        save("rd", rdh);

        // step 4: power, alpha, CA-CFAR
        std::vector<float> power(rdh.size());
        for (std::size_t i = 0; i < rdh.size(); ++i) power[i] = rdh[i].re * rdh[i].re + rdh[i].im * rdh[i].im;
        save("power", power);
        auto dpower = DeviceArray<float>::from_host(power);
        CaCfarOptions co;
        co.guard_cells = {2, 2};
        co.reference_cells = {4, 4};
        co.pfa = 1e-3;
        auto alpha = cfar_alpha_device<float>(1e-3f, 2 * 4 * (2 * 4 + 2 * 2 + 1) + 2 * (2 * 2 + 1) * 4);
        save("alpha", alpha.to_host());
        auto cf = ca_cfar_device(dpower, {P, N}, co);
        save("thr", cf.threshold.to_host());
        save("det", cf.detections.to_host());
        set_ca_cfar_device_method(CaCfarDeviceMethod::fp64_decided);
        auto cf64 = ca_cfar_device(dpower, {P, N}, co);
        set_ca_cfar_device_method(CaCfarDeviceMethod::reference_order);
        save("det64", cf64.detections.to_host());

        // integer CFAR input (floor rule) and half-precision compression input
        auto ipow = DeviceArray<std::int16_t>::from_host(load<std::int16_t>("ipow.bin"));
        auto cfi = ca_cfar_device(ipow, {P, N}, co);
        save("ithr", cfi.threshold.to_host());
        save("idet", cfi.detections.to_host());
        auto xh = DeviceArray<TypedComplex<__half>>::from_host(load<TypedComplex<__half>>("xh.bin"));
        auto th = DeviceArray<TypedComplex<__half>>::from_host(load<TypedComplex<__half>>("th.bin"));
        auto comph = pulse_compression_device(xh, th, pc);
        save("pch", comph.fp32.to_host());

        // front end: firfilter (1-D and 2-D along axis 0), upfirdn, resample_poly
        auto b = DeviceArray<float>::from_host(load<float>("b.bin"));
        auto s = DeviceArray<float>::from_host(load<float>("s.bin"));
        FirfilterDeviceResult fr;
        firfilter_device(b, s, fr);
        save("fir", fr.y.to_host());
        DeviceArray<float> yres(s.size());
        firfilter_fp32_resident_device(b, s, yres);
        save("fir_resident", yres.to_host());
        FirfilterOptions fo;
        fo.shape = {NF / 4, 4};
        fo.axis = 0;
        FirfilterDeviceResult fr2;
        firfilter_device(b, s, fr2, fo);
        save("fir_axis0", fr2.y.to_host());
        auto h = DeviceArray<float>::from_host(load<float>("h.bin"));
        UpfirdnDeviceResult ur;
        upfirdn_device(h, s, 3, 2, ur);
        save("upfirdn", ur.fp32.to_host());
        ResamplePolyDeviceResult rr;
        resample_poly_device(s, 3, 2, rr);
        if (rr.dtype != ResamplePolyOutputDtype::fp64) throw std::runtime_error("default design stores FP64");
        save("resample", rr.fp64.to_host());
        auto si = DeviceArray<std::int16_t>::from_host(load<std::int16_t>("si.bin"));
        auto hi = DeviceArray<std::int16_t>::from_host(load<std::int16_t>("hi.bin"));
        UpfirdnDeviceResult uri;
        upfirdn_device(hi, si, 2, 3, uri);
        save("upfirdn_i16", uri.fp32.to_host());

        // zero-phase FIR (default odd padding; int16 with even padding along axis 0) and the
        // analytic signal (length 5000, and an int16 input along axis 0)
        Firfilter2DeviceResult f2;
        firfilter2_device(b, s, f2);
        if (f2.dtype != Firfilter2OutputDtype::fp32) throw std::runtime_error("firfilter2 of float is FP32");
        save("fir2", f2.fp32.to_host());
        auto b16 = DeviceArray<std::int16_t>::from_host(std::vector<std::int16_t>{1, 2, 1});
        Firfilter2Options f2o;
        f2o.shape = {NF / 8, 8};
        f2o.axis = 0;
        f2o.padtype = Firfilter2PadType::even;
        f2o.padlen = 20;
        Firfilter2DeviceResult f2i;
        firfilter2_device(b16, si, f2i, f2o);
        save("fir2_i16_axis0", f2i.fp32.to_host());
        bool gust_threw = false;
        try {
            Firfilter2Options g;
            g.method = Firfilter2Method::gust;
            Firfilter2DeviceResult bad;
            firfilter2_device(b, s, bad, g);
        } catch (const std::invalid_argument&) {
            gust_threw = true;
        }
        if (!gust_threw) throw std::runtime_error("firfilter2 gust did not throw");
        HilbertOptions ho;
        ho.fft_length = 5000;
        HilbertDeviceResult hr;
        hilbert_device(s, hr, ho);
        if (hr.dtype != HilbertOutputDtype::complex_fp32 || hr.shape[0] != 5000)
            throw std::runtime_error("hilbert of float is ComplexFP32 [N]");
        save("hilbert", hr.complex_fp32.to_host());
        HilbertOptions hio;
        hio.shape = {NF / 8, 8};
        hio.axis = 0;
        HilbertDeviceResult hri;
        hilbert_device(si, hri, hio);
        if (hri.dtype != HilbertOutputDtype::complex_fp64) throw std::runtime_error("hilbert of int16 is ComplexFP64");
        save("hilbert_i16_axis0", hri.complex_fp64.to_host());

        // batched FFT round trip
        FFTInterface fft(N, FFTInterface::BatchOnly{});
        DeviceArray<ComplexFloat> spec(static_cast<std::size_t>(P) * N), back(static_cast<std::size_t>(P) * N);
        fft.fft_batch_device(reinterpret_cast<const ComplexFloat*>(x.data()), spec.data(), P, x.size());
        fft.ifft_batch_device(spec, back, P);
        save("fft", spec.to_host());
        save("ifft", back.to_host());

        // ambiguity function of the template, the calls Task1 step 5 makes
        AmbgfunOptions ao;
        ao.fs = 2.0;
        ao.prf = 1.0;
        AmbgfunDeviceResult a2d, adelay, adoppler;
        ambgfun_device<float>(t, a2d, ao);
        if (a2d.dtype != AmbgfunOutputDtype::fp32) throw std::runtime_error("2-D ambgfun of float is FP32");
        save("amb2d", a2d.fp32.to_host());
        ao.cut = AmbgfunCut::doppler;
        ao.cut_value = 0.1;
        ambgfun_device<float>(t, adoppler, ao);
        save("ambdoppler", adoppler.fp64.to_host());
        ao.cut = AmbgfunCut::delay;
        ao.cut_value = 3.0;
        ambgfun_device<float>(t, adelay, ao);
        save("ambdelay", adelay.fp64.to_host());
        bool amb_threw = false;
        try {
            ao.fs = 0.0;
            AmbgfunDeviceResult bad;
            ambgfun_device<float>(t, bad, ao);
        } catch (const std::invalid_argument&) {
            amb_threw = true;
        }
        if (!amb_threw) throw std::runtime_error("ambgfun with fs = 0 did not throw");

        // error contract: invalid shapes throw std::invalid_argument
        bool threw = false;
        try {
            PulseCompressionOptions bad = pc;
            bad.num_pulses = 0;
            (void)pulse_compression_device(x, t, bad);
        } catch (const std::invalid_argument&) {
            threw = true;
        }
        if (!threw) throw std::runtime_error("invalid shape did not throw std::invalid_argument");
        (void)NT;
        std::cout << "dropin ok\n";
        return 0;
    } catch (const std::exception& e) {
        std::cerr << "dropin failed: " << e.what() << "\n";
        return 1;
    }
}
