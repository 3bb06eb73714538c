// lpaici_cli.cpp -- drop-in command line for the reference executables (titocapovilla/lpa-ici-cuda):
// the same options and defaults (src/Config.hpp:7-92), the same outputs (gray_image.hdr and
// gray_image_noisy.hdr next to the -o file, and the denoised .hdr) and the same stdout lines as the
// reference's fastest GPU executable (main of src/v4_1_lpa_ici_2D_sparse_shared.cu:365-530),
// computed by the B200 library through its C ABI.
//
//   lpaici [-i image] [-k kernels] [-o output.hdr] [-s sigma(0-255)] [-g gamma] [--seed n] [--color] [-h]
//
// --color (not in the reference, which converts every image to gray) keeps the image's R, G and B
// channels, adds noise to all of them and denoises each channel on its own; its files are
// color_image.hdr, color_image_noisy.hdr and the RGB -o file, its PSNR lines cover all channels.
//
// Errors print a message and exit with status 1, as the reference does; nothing here calls exit()
// from inside the library.
#include <chrono>
#include <cstdlib>
#include <iostream>
#include <string>
#include <vector>

#include "image_io.h"
#include "lpaici.h"

namespace {

const char *kVersion = "lpaici_b200_gpu";

struct Config {
    std::string image_file = "data/barbara.png";
    std::string kernel_file = "kernels/lpa_kernels_m_1_0_d_16_h12_1_2_4_8_16_24_32_symmetric.txt";
    std::string output_file;  // empty: <image dir>/<image name>_<version>.hdr
    float sigma_noise = 20.0f / 255.0f;
    unsigned int noise_seed = 20250910u;
    float ici_gamma = 2.0f;
    bool color = false;
};

std::string dir_of(const std::string &path) {
    const size_t slash = path.find_last_of('/');
    return slash == std::string::npos ? "" : path.substr(0, slash + 1);
}

void usage(const char *prog) {
    const Config d;
    std::cout << "Usage: " << prog << " [options]\n"
              << "  -i, --image <file>     input image (default " << d.image_file << ")\n"
              << "  -k, --kernels <file>   LPA kernel file, text or binary tap-list (default " << d.kernel_file << ")\n"
              << "  -o, --output <file>    denoised .hdr output (default <image dir>/<image name>_<version>.hdr)\n"
              << "  -s, --sigma <value>    noise standard deviation on the 0-255 scale (default 20)\n"
              << "  -g, --gamma <value>    ICI threshold (default " << d.ici_gamma << ")\n"
              << "      --seed <value>     noise seed (default " << d.noise_seed << ")\n"
              << "      --color            denoise the R, G, B channels (default: gray, as the reference)\n"
              << "  -h, --help             show this message\n";
}

[[noreturn]] void fail(const char *prog, const std::string &msg) {
    std::cerr << "Error: " << msg << "\n\n";
    usage(prog);
    std::exit(EXIT_FAILURE);
}

Config parse(int argc, char **argv) {
    Config cfg;
    auto positive = [&](const std::string &opt, const char *s) {
        char *end = nullptr;
        const float v = std::strtof(s, &end);
        if (*s == '\0' || *end != '\0' || !(v > 0.0f)) fail(argv[0], opt + " needs a positive number, got '" + s + "'");
        return v;
    };
    for (int i = 1; i < argc; i++) {
        const std::string opt = argv[i];
        if (opt == "-h" || opt == "--help") {
            usage(argv[0]);
            std::exit(EXIT_SUCCESS);
        }
        if (opt == "--color") {
            cfg.color = true;
            continue;
        }
        if (i + 1 >= argc) fail(argv[0], "unknown option or missing value for '" + opt + "'");
        const char *val = argv[++i];
        if (opt == "-i" || opt == "--image") {
            cfg.image_file = val;
        } else if (opt == "-k" || opt == "--kernels") {
            cfg.kernel_file = val;
        } else if (opt == "-o" || opt == "--output") {
            cfg.output_file = val;
        } else if (opt == "-s" || opt == "--sigma") {
            cfg.sigma_noise = positive(opt, val) / 255.0f;
        } else if (opt == "-g" || opt == "--gamma") {
            cfg.ici_gamma = positive(opt, val);
        } else if (opt == "--seed") {
            char *end = nullptr;
            const unsigned long v = std::strtoul(val, &end, 10);
            if (*val == '\0' || *end != '\0') fail(argv[0], "--seed needs an unsigned integer, got '" + std::string(val) + "'");
            cfg.noise_seed = static_cast<unsigned int>(v);
        } else {
            fail(argv[0], "unknown option '" + opt + "'");
        }
    }
    if (cfg.output_file.empty()) {
        std::string name = cfg.image_file.substr(dir_of(cfg.image_file).size());
        name = name.substr(0, name.find_last_of('.'));
        cfg.output_file = dir_of(cfg.image_file) + name + "_" + kVersion + ".hdr";
    }
    std::cout << "Image: " << cfg.image_file << "\n"
              << "Kernels: " << cfg.kernel_file << "\n"
              << "Output: " << cfg.output_file << "\n"
              << "Sigma: " << cfg.sigma_noise * 255.0f << "/255, gamma: " << cfg.ici_gamma
              << ", seed: " << cfg.noise_seed << "\n";
    return cfg;
}

}  // namespace

int main(int argc, char **argv) {
    const Config cfg = parse(argc, argv);

    std::vector<float> clean;
    int width = 0, height = 0;
    std::string err;
    const int channels = cfg.color ? 3 : 1;
    if (!lpaici_cli::load_image(cfg.image_file, channels, clean, width, height, err)) {
        std::cerr << "Error in loading the image " << cfg.image_file << "\n";
        return 1;
    }
    std::cout << "Loaded image with a width of " << width << " px, a height of " << height
              << " px and (imported) " << channels << " channels\n";

    const std::string kind = cfg.color ? "color" : "gray";
    const std::string gray_file = dir_of(cfg.output_file) + kind + "_image.hdr";
    std::cout << "Saving " << kind << " image as " << gray_file << "\n";
    lpaici_cli::write_hdr(gray_file, clean.data(), width, height, channels);

    const long n = static_cast<long>(width) * height * channels;
    std::vector<float> noisy(n);
    lpaici_add_noise(clean.data(), noisy.data(), n, cfg.sigma_noise, cfg.noise_seed);
    const std::string noisy_file = dir_of(cfg.output_file) + kind + "_image_noisy.hdr";
    std::cout << "Saving noisy " << kind << " image as " << noisy_file << "\n";
    lpaici_cli::write_hdr(noisy_file, noisy.data(), width, height, channels);

    const double psnr_noisy = lpaici_psnr(clean.data(), noisy.data(), n);
    std::cout << "Calculated PSNR of host_img_gray_noisy: " << psnr_noisy << "\n";

    lpaici_kernelset *ks = nullptr;
    int rc = lpaici_kernelset_load(cfg.kernel_file.c_str(), &ks);
    if (rc != LPAICI_OK) {
        std::cerr << "Error: " << lpaici_last_error() << std::endl;
        return 1;
    }
    lpaici_kernelset_info_t info{};
    lpaici_kernelset_get_info(ks, &info);
    const int nk = info.num_dirs * info.num_scales;
    std::vector<float> weights(info.dense_size);
    std::vector<int> offsets(nk), rows(nk), cols(nk);
    lpaici_kernelset_get_dense(ks, weights.data(), offsets.data(), rows.data(), cols.data());
    std::cout << "Precomputing kernel variances \n";
    std::vector<float> variances(nk);
    lpaici_kernel_variances(ks, cfg.sigma_noise, variances.data());

    std::vector<float> denoised(n, 0.0f);
    const auto t0 = std::chrono::steady_clock::now();
    std::cout << "Executing LPA ICI fused algorithm \n";
    double loop_seconds = 0.0;
    rc = lpaici_anisotropic_gpu_fused(noisy.data(), denoised.data(), width, height, channels, nullptr,
                                      info.num_dirs, info.num_scales, weights.data(), info.dense_size, offsets.data(),
                                      rows.data(), cols.data(), variances.data(), cfg.ici_gamma, &loop_seconds);
    if (rc != LPAICI_OK) {
        std::cerr << "Error: " << lpaici_last_error() << std::endl;
        lpaici_kernelset_destroy(ks);
        return 1;
    }
    std::cout << "Time taken for directional loops + aggregation: " << loop_seconds << " seconds\n";
    const double total = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    std::cout << "Time taken for lpa function execution: " << total << " seconds\n";

    const double psnr_denoised = lpaici_psnr(clean.data(), denoised.data(), n);
    std::cout << "Calculated PSNR of img_denoised: " << psnr_denoised << "\n";
    std::cout << "Saving denoised image as " << cfg.output_file.c_str() << "\n";
    lpaici_cli::write_hdr(cfg.output_file, denoised.data(), width, height, channels);

    lpaici_kernelset_destroy(ks);
    return 0;
}
