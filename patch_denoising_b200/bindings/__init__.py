"""Front-end bindings: method registry, configuration strings, command line."""
