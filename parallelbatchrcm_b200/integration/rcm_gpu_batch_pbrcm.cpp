// rcm_gpu_batch_pbrcm.cpp -- GPU_BATCH::rcm / GPU_BATCH::findPeripheral of the
// reference (include/rcm_gpu_batch.h:40-44 there) implemented on libpbrcm.
//
// This file is the shim a maintainer compiles into the reference in place of
// src/device/rcm_gpu_batch.cu: it includes the reference's own headers
// (Graph.h, rcm_gpu_batch.h) and calls the C ABI of include/pbrcm.h.  Same
// signature, same output (the Cuthill-McKee order from the given start, not
// reversed, as the reference returns it), same timing line on stdout and in
// the CSV file, same exception type on failure.
#include "rcm_gpu_batch.h"

#include <iomanip>
#include <iostream>
#include <stdexcept>
#include <string>

#include "pbrcm.h"

namespace GPU_BATCH
{
	template<typename T>
	void rcm(Graph<T>& graph, std::ofstream& csv_file, std::vector<unsigned>& permutation, unsigned start_node)
	{
		pbrcm_options opts;
		pbrcm_default_options(&opts);
		opts.reverse = 0;
		opts.start_node = start_node;
		opts.want_bandwidth = 0;
		permutation.resize(graph.csr.rows);
		pbrcm_result res;
		int32_t rc = pbrcm_reorder(nullptr, graph.csr.row_offsets.get(), graph.csr.col_ids.get(),
		                           static_cast<uint32_t>(graph.csr.rows), graph.csr.nnz, &opts,
		                           permutation.data(), &res);
		if (rc != PBRCM_OK)
			throw std::runtime_error(std::string("CUDA ERROR: ") + pbrcm_status_string(rc));
		std::cout << std::setw(27) << std::right << "GPU-DYN-RCM" << " duration: " << res.device_ms << " ms" << std::endl;
		csv_file << res.device_ms;
		csv_file << std::flush;
	}

	template<typename T>
	void findPeripheral(Graph<T>& graph, std::ofstream& csv_file, bool writeOutput)
	{
		uint32_t start = 0, passes = 0, ecc = 0;
		int32_t rc = pbrcm_find_peripheral(nullptr, graph.csr.row_offsets.get(), graph.csr.col_ids.get(),
		                                   static_cast<uint32_t>(graph.csr.rows), graph.csr.nnz, &start, &passes,
		                                   &ecc);
		if (rc != PBRCM_OK)
			throw std::runtime_error(std::string("CUDA ERROR: ") + pbrcm_status_string(rc));
		std::cout << std::setw(27) << std::right << ("Opt-GPU-Peripheral<" + std::to_string(passes) + ", " +
		                                             std::to_string(start) + ", " + std::to_string(ecc) + ">")
		          << std::endl;
		if (writeOutput)
			csv_file << "," << 0 << std::flush;
	}

	template void rcm(Graph<float>& graph, std::ofstream& csv_file, std::vector<unsigned>& permutation, unsigned start_node);
	template void rcm(Graph<double>& graph, std::ofstream& csv_file, std::vector<unsigned>& permutation, unsigned start_node);
	template void findPeripheral(Graph<float>& graph, std::ofstream& csv_file, bool writeOutput);
	template void findPeripheral(Graph<double>& graph, std::ofstream& csv_file, bool writeOutput);
}
