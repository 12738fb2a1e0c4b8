/*
 * Test infrastructure (oracle), not product code.
 *
 * In-memory stand-in for the reference's `nbl::hdf5_file`
 * (io/hdf5_file.h:27-177), used only to compile the reference's own CPU
 * driver and its octree/physics headers here, where HDF5 is not installed.
 * It is force-included (`g++ -include`) before the reference sources and
 * defines the reference's include guard `__HDF5_FILE_H_`, so the real
 * header (and its libhdf5 dependency) drops out.
 *
 * It serves the same content an HDF5 material file holds -- quantity
 * properties with units, float datasets with per-axis dimension scales and a
 * `units` attribute -- read from a `.nmat` file (format documented in
 * nebula_b200/synth/nmat.py).  The member functions keep the reference's
 * signatures and semantics:
 *   - get_property_quantity: value * parsed unit; the defaulted overload
 *     returns the default when the property is absent (hdf5_file.cpp:188-227);
 *   - fill_table1D/2D/3D: table created over [0,1] and filled row-major
 *     (hdf5_file.cpp:229-287);
 *   - get_lin_dimscale / get_log_dimscale: linspace / geomspace of the scale's
 *     first and last values times its unit; a missing linear scale gives
 *     [0,1] (hdf5_file.cpp:289-358);
 *   - get_unit: the dataset's unit string parsed (hdf5_file.cpp:361-375).
 */
#ifndef NBL_ORACLE_HDF5_STANDIN_H
#define NBL_ORACLE_HDF5_STANDIN_H

#include "config/config.h"

#define __HDF5_FILE_H_

#include <string>
#include <vector>
#include <map>
#include <fstream>
#include <stdexcept>
#include <cstring>
#include <cstdint>
#include "common/units/unit_system.h"
#include "common/util/range.h"
#include "common/util/table_1D.h"
#include "common/util/table_2D.h"
#include "common/util/table_3D.h"

namespace nbl {

class hdf5_file
{
public:
	hdf5_file(std::string const & filename) : _filename(filename)
	{
		std::ifstream f(filename, std::ios::binary);
		if (!f)
			throw std::runtime_error("Unable to open file " + filename);
		std::vector<char> buf((std::istreambuf_iterator<char>(f)), std::istreambuf_iterator<char>());
		size_t off = 0;
		auto need = [&](size_t n) {
			if (off + n > buf.size())
				throw std::runtime_error("Truncated material file " + filename);
		};
		auto u32 = [&]() { need(4); uint32_t v; std::memcpy(&v, buf.data() + off, 4); off += 4; return v; };
		auto u64 = [&]() { need(8); uint64_t v; std::memcpy(&v, buf.data() + off, 8); off += 8; return v; };
		auto f64 = [&]() { need(8); double v; std::memcpy(&v, buf.data() + off, 8); off += 8; return v; };
		auto str = [&]() { uint32_t n = u32(); need(n); std::string s(buf.data() + off, n); off += n; return s; };

		need(8);
		if (std::memcmp(buf.data(), "NBLMAT01", 8) != 0)
			throw std::runtime_error("Not a material file: " + filename);
		off = 8;
		uint32_t np = u32();
		for (uint32_t i = 0; i < np; ++i)
		{
			std::string name = str();
			double value = f64();
			std::string unit = str();
			_props[name] = std::make_pair(value, unit);
		}
		uint32_t nd = u32();
		for (uint32_t i = 0; i < nd; ++i)
		{
			dataset d;
			std::string name = str();
			d.unit = str();
			uint32_t ndim = u32();
			for (uint32_t a = 0; a < ndim; ++a)
				d.dims.push_back(u64());
			for (uint32_t a = 0; a < ndim; ++a)
			{
				need(1);
				char has = buf[off++];
				scale s;
				s.present = has != 0;
				if (s.present)
				{
					s.unit = str();
					s.values.resize(d.dims[a]);
					need(8 * d.dims[a]);
					std::memcpy(s.values.data(), buf.data() + off, 8 * d.dims[a]);
					off += 8 * d.dims[a];
				}
				d.scales.push_back(s);
			}
			size_t count = 1;
			for (auto n : d.dims)
				count *= n;
			d.data.resize(count);
			need(4 * count);
			std::memcpy(d.data.data(), buf.data() + off, 4 * count);
			off += 4 * count;
			_sets[canonical(name)] = d;
		}
	}

	// HDF5 resolves "a/b" and "/a/b" alike (the reference asks for both
	// forms, e.g. kieft/inelastic.h:263 and full_penn.h:374)
	static std::string canonical(std::string const & name)
	{
		size_t i = 0;
		while (i < name.size() && name[i] == '/')
			++i;
		return name.substr(i);
	}

	std::string const & get_filename() const { return _filename; }

	bool exists(std::string const & query) const
	{
		const std::string name = canonical(query);
		if (_sets.count(name))
			return true;
		// group paths ("/elastic") exist when a dataset lives under them
		for (auto const & kv : _sets)
			if (kv.first.compare(0, name.size(), name) == 0 &&
				kv.first.size() > name.size() && kv.first[name.size()] == '/')
				return true;
		return false;
	}

	std::string get_property_string(std::string const & name) const
	{
		auto it = _props.find(name);
		if (it == _props.end())
			throw std::runtime_error("Could not read string property '" + name + '\'');
		return it->second.second;
	}
	units::quantity<double> get_property_quantity(std::string const & name,
		units::unit_parser<double> const & parser = units::default_unit_parser()) const
	{
		auto it = _props.find(name);
		if (it == _props.end())
			throw std::runtime_error("Could not read quantity property '" + name + '\'');
		return it->second.first * parser.parse_unit(it->second.second);
	}
	std::string get_property_string(std::string const & name, std::string const & _default) const
	{
		auto it = _props.find(name);
		return it == _props.end() ? _default : it->second.second;
	}
	units::quantity<double> get_property_quantity(std::string const & name,
		units::quantity<double> const & _default,
		units::unit_parser<double> const & parser = units::default_unit_parser()) const
	{
		auto it = _props.find(name);
		if (it == _props.end())
			return _default;
		return it->second.first * parser.parse_unit(it->second.second);
	}

	template<typename T>
	util::table_1D<T, false> fill_table1D(std::string const & dataset_name) const
	{
		dataset const & d = get(dataset_name, 1);
		auto table = util::table_1D<T, false>::create(0, 1, int(d.dims[0]));
		T* out = table.data();
		for (size_t i = 0; i < d.data.size(); ++i)
			out[i] = static_cast<T>(d.data[i]);
		return table;
	}
	template<typename T>
	util::table_2D<T, false> fill_table2D(std::string const & dataset_name) const
	{
		dataset const & d = get(dataset_name, 2);
		auto table = util::table_2D<T, false>::create(0, 1, int(d.dims[0]), 0, 1, int(d.dims[1]));
		T* out = table.data();
		for (size_t i = 0; i < d.data.size(); ++i)
			out[i] = static_cast<T>(d.data[i]);
		return table;
	}
	template<typename T>
	util::table_3D<T, false> fill_table3D(std::string const & dataset_name) const
	{
		dataset const & d = get(dataset_name, 3);
		auto table = util::table_3D<T, false>::create(0, 1, int(d.dims[0]),
			0, 1, int(d.dims[1]), 0, 1, int(d.dims[2]));
		T* out = table.data();
		for (size_t i = 0; i < d.data.size(); ++i)
			out[i] = static_cast<T>(d.data[i]);
		return table;
	}

	util::linspace<units::quantity<double>> get_lin_dimscale(std::string const & dataset_name,
		int dim, int N_expected,
		units::unit_parser<double> const & parser = units::default_unit_parser()) const
	{
		dataset const & d = get(dataset_name, -1);
		scale const & s = d.scales.at(dim);
		if (!s.present)
			return util::linspace<units::quantity<double>>(0*units::dimensionless, 1*units::dimensionless, N_expected);
		if (s.values.size() != (size_t)N_expected)
			throw std::runtime_error("Dimension scale has unexpected size.");
		const auto unit = parser.parse_unit(s.unit);
		return util::linspace<units::quantity<double>>(s.values.front() * unit, s.values.back() * unit, N_expected);
	}
	util::geomspace<units::quantity<double>> get_log_dimscale(std::string const & dataset_name,
		int dim, int N_expected,
		units::unit_parser<double> const & parser = units::default_unit_parser()) const
	{
		dataset const & d = get(dataset_name, -1);
		scale const & s = d.scales.at(dim);
		if (!s.present || s.values.size() != (size_t)N_expected)
			throw std::runtime_error("Dimension scale has unexpected size.");
		const auto unit = parser.parse_unit(s.unit);
		return util::geomspace<units::quantity<double>>(s.values.front() * unit, s.values.back() * unit, N_expected);
	}

	units::quantity<double> get_unit(std::string const & dataset_name,
		units::unit_parser<double> const & parser = units::default_unit_parser()) const
	{
		return parser.parse_unit(get(dataset_name, -1).unit);
	}

private:
	struct scale { bool present = false; std::string unit; std::vector<double> values; };
	struct dataset { std::string unit; std::vector<uint64_t> dims; std::vector<scale> scales; std::vector<float> data; };

	dataset const & get(std::string const & name, int ndim) const
	{
		auto it = _sets.find(canonical(name));
		if (it == _sets.end())
			throw std::runtime_error("Could not read table '" + name + '\'');
		if (ndim >= 0 && it->second.dims.size() != (size_t)ndim)
			throw std::runtime_error("Table '" + name + "' has the wrong rank");
		return it->second;
	}

	std::string _filename;
	std::map<std::string, std::pair<double, std::string>> _props;
	std::map<std::string, dataset> _sets;
};

} // namespace nbl

#endif // NBL_ORACLE_HDF5_STANDIN_H
