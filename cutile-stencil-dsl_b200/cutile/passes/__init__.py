"""Analysis and optimization passes over Dialect 2."""
