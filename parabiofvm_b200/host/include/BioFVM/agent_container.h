// Agent containers (include/BioFVM/agent_container_base.h and src/agent_container.h of the
// reference): agents are objects pointing into shared structure-of-arrays storage; removing one
// moves the last agent into its slot, in the storage and in the object list alike.
#pragma once

#include <memory>
#include <type_traits>
#include <utility>
#include <vector>

#include "agent.h"
#include "agent_data.h"

namespace biofvm {

namespace solvers::b200 {
class solver;
class cell_solver;
}

class agent_container_base;
using agent_ptr = std::unique_ptr<agent>;
using agent_container_ptr = std::unique_ptr<agent_container_base>;

class agent_container_base
{
	friend solvers::b200::solver;
	friend solvers::b200::cell_solver;

protected:
	virtual agent_data& get_agent_data() = 0;

	agent_id_t next_agent_id_ = 0;

	agent_container_base() = default;

	static index_t& get_agent_index(agent* a) { return a->index_; }

public:
	virtual index_t agents_count() const = 0;
	virtual agent* create_agent() = 0;
	virtual void remove_agent(agent* a) = 0;
	virtual void remove_at(index_t index) = 0;
	virtual agent* get_agent_at(index_t index) = 0;

	virtual ~agent_container_base() = default;
};

template <typename agent_t, typename agent_data_t>
class agent_container_common : public agent_container_base
{
protected:
	agent_data_t data_;
	std::vector<std::unique_ptr<agent_t>> agents_;

	template <typename... args_t>
	explicit agent_container_common(args_t&&... args) : data_(std::forward<args_t>(args)...)
	{}

	agent_data& get_agent_data() override { return data_; }

public:
	index_t agents_count() const override { return (index_t)agents_.size(); }

	agent* create_agent() override { return create(); }

	template <typename other_agent_t = agent_t>
	other_agent_t* create()
	{
		data_.add();
		auto made = std::make_unique<other_agent_t>(next_agent_id_++, data_, data_.agents_count - 1);
		other_agent_t* raw = made.get();
		agents_.push_back(std::move(made));
		return raw;
	}

	void remove_agent(agent* a) override { remove_at(get_agent_index(a)); }

	void remove_at(index_t index) override
	{
		// the last agent takes the freed slot
		get_agent_index(agents_.back().get()) = index;
		std::swap(agents_[index], agents_.back());
		agents_.pop_back();
		data_.remove(index);
	}

	agent* get_agent_at(index_t index) override { return get_at(index); }

	template <typename other_agent_t = agent_t>
	other_agent_t* get_at(index_t index)
	{
		if constexpr (std::is_same_v<other_agent_t, agent_t>)
			return agents_[index].get();
		else
			return dynamic_cast<other_agent_t*>(agents_[index].get());
	}

	const std::vector<std::unique_ptr<agent_t>>& agents() const { return agents_; }
	const agent_data_t& data() const { return data_; }
};

struct microenvironment;

class agent_container : public agent_container_common<agent, agent_data>
{
public:
	explicit agent_container(microenvironment& m) : agent_container_common(m) {}
};

} // namespace biofvm
