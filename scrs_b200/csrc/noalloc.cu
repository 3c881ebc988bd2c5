// (reserved)
